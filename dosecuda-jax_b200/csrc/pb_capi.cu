// pb_capi.cu -- the extern "C" entry points of libpb_b200.so: argument
// checks, host-side plan preparation and the host-buffer drop-in level.
//
// Host preparation follows the reference:
//   beam set-up              DoseCUDA/dose_kernels/dosemodule.cu:148-175,
//                            CudaClasses.cu:17-51
//   spot sort + layers       dosemodule.cu:204-225, IMPTClasses.cu:29-67
// The drop-in level replaces IMPTClasses.cu:274-340 (proton_raytrace_cuda,
// proton_spot_cuda); unlike the reference it keeps its device buffers
// between calls (grow-only, per device) instead of allocating and freeing
// every buffer on every call.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "pb_internal.h"

namespace pb {

static thread_local std::string g_err;

PbStatus set_error(PbStatus code, const char *fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

PbStatus check_cuda(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return PB_OK;
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        return set_error(PB_ERR_NOMEM, "%s: %s", what, cudaGetErrorString(e));
    }
    return set_error(PB_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

PbStatus check_launch(const char *what) { return check_cuda(cudaGetLastError(), what); }

void smooth_dirs(float *c, float *s)
{
    for (int i = 0; i < 6; ++i) {
        // volatile keeps the compiler from folding sinf/cosf at build time:
        // the values must be the C library's, as the oracle computes them.
        volatile float a = (float)i * 3.141592654f / 3.0f;
        c[i] = cosf(a);
        s[i] = sinf(a);
    }
}

static PbStatus check_grid(const PbGrid *g)
{
    if (!g) return set_error(PB_ERR_INVALID, "grid is NULL");
    if (g->nx <= 0 || g->ny <= 0 || g->nz <= 0)
        return set_error(PB_ERR_INVALID, "grid dimensions must be positive (got %d x %d x %d)",
                         g->nx, g->ny, g->nz);
    const int64_t v = (int64_t)g->nx * g->ny * g->nz;
    if (v > (int64_t)INT32_MAX)
        return set_error(PB_ERR_INVALID, "grid has %lld voxels; at most %d supported",
                         (long long)v, INT32_MAX);
    if (!(g->spacing > 0.0f) || !std::isfinite(g->spacing))
        return set_error(PB_ERR_INVALID, "spacing must be a positive finite number");
    return PB_OK;
}

static PbStatus check_beams(const PbGrid *g, const PbBeam *beams, int n_beams,
                            const float *wet, const PbLayer *layers, const float *geo,
                            bool need_geo = true)
{
    PbStatus s = check_grid(g);
    if (s != PB_OK) return s;
    if (!beams || n_beams <= 0 || n_beams > PB_MAX_BEAMS)
        return set_error(PB_ERR_INVALID, "n_beams must be in [1, %d] (got %d)", PB_MAX_BEAMS,
                         n_beams);
    if (!wet) return set_error(PB_ERR_INVALID, "wet is NULL");
    for (int b = 0; b < n_beams; ++b) {
        const PbBeam &B = beams[b];
        if (B.n_layers < 0 || B.layer_start < 0 || B.spot_start < 0 || B.n_spots < 0)
            return set_error(PB_ERR_INVALID, "beam %d: negative layer/spot range", b);
        if (B.n_layers == 0) continue;
        if (!layers || (need_geo && !geo))
            return set_error(PB_ERR_INVALID, "layers/spot geometry is NULL");
        if (!B.dvp_dev || !B.depths_dev || !B.sigmas_dev || !B.idds_dev)
            return set_error(PB_ERR_INVALID, "beam %d: model table is NULL", b);
        if (B.lut_len <= 0 || B.lut_len > PB_MAX_LUT_LEN)
            return set_error(PB_ERR_INVALID, "beam %d: lut_len must be in [1, %d] (got %d)", b,
                             PB_MAX_LUT_LEN, B.lut_len);
        if (B.dvp_len < 5)
            return set_error(PB_ERR_INVALID, "beam %d: dvp_len must be >= 5 (got %d)", b,
                             B.dvp_len);
        if (B.n_energies <= 0) return set_error(PB_ERR_INVALID, "beam %d: no energies", b);
    }
    return PB_OK;
}

PbStatus check_wet_args(const float *rlsp_dev, uint64_t tex, const PbGrid *grid,
                        const PbBeamGeom *beams, int n_beams, const float *wet_dev)
{
    PbStatus s = check_grid(grid);
    if (s != PB_OK) return s;
    if ((!rlsp_dev && !texture_samples(tex)) || !beams || !wet_dev)
        return set_error(PB_ERR_INVALID, "NULL argument");
    if (tex && !texture_matches(tex, *grid))
        return set_error(PB_ERR_INVALID, "texture extent differs from the grid");
    if (n_beams <= 0 || n_beams > PB_MAX_BEAMS)
        return set_error(PB_ERR_INVALID, "n_beams must be in [1, %d] (got %d)", PB_MAX_BEAMS,
                         n_beams);
    return PB_OK;
}

}  // namespace pb

using namespace pb;

extern "C" {

const char *pb_last_error(void) { return g_err.c_str(); }

const char *pb_version(void) { return "pb_b200 1.0 (sm_100a)"; }

PbStatus pb_beam_setup(double gantry_deg, double couch_deg, double vsadx, double vsady,
                       const float iso[3], const float origin[3], PbBeamGeom *out)
{
    if (!iso || !origin || !out) return set_error(PB_ERR_INVALID, "NULL argument");
    const float pi_f = 3.141592654f;
    const float ga = fmodf((float)(gantry_deg + 180.0), 360.0f);
    const float ta = (float)couch_deg;
    const float gar = ga * pi_f / 180.0f;
    const float tar = ta * pi_f / 180.0f;
    out->singa = sinf(gar);
    out->cosga = cosf(gar);
    out->sinta = sinf(tar);
    out->costa = cosf(tar);
    out->vsadx = (float)vsadx;
    out->vsady = (float)vsady;
    const float sd = (out->vsadx + out->vsady) / 2.0f;
    const float xg = -sd * out->singa;
    const float yg = sd * out->cosga;
    out->src[0] = xg * out->costa;
    out->src[1] = yg;
    out->src[2] = -xg * out->sinta;
    for (int d = 0; d < 3; ++d) out->iso[d] = iso[d] - origin[d];
    return PB_OK;
}

PbStatus pb_build_layers(const float *spot_list, int n_spots, const float *dvp, int dvp_len,
                         int n_energies, PbSpot *spots_out, PbLayer *layers_out,
                         int *n_layers_out, int *perm_out)
{
    if (n_spots < 0 || n_energies < 0 || dvp_len < 2)
        return set_error(PB_ERR_INVALID, "invalid spot/energy counts");
    if ((n_spots > 0 && (!spot_list || !spots_out)) || !n_layers_out ||
        (n_energies > 0 && (!dvp || !layers_out)))
        return set_error(PB_ERR_INVALID, "NULL argument");
    std::vector<int> order((size_t)n_spots);
    std::vector<int> eid((size_t)n_spots);
    for (int q = 0; q < n_spots; ++q) {
        order[q] = q;
        eid[q] = static_cast<int>(spot_list[4 * (size_t)q + 3]);
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return eid[a] < eid[b]; });
    for (int q = 0; q < n_spots; ++q) {
        const int o = order[q];
        spots_out[q].x = spot_list[4 * (size_t)o];
        spots_out[q].y = spot_list[4 * (size_t)o + 1];
        spots_out[q].mu = spot_list[4 * (size_t)o + 2];
        spots_out[q].energy_id = eid[o];
        if (perm_out) perm_out[q] = o;
    }
    // importLayers: walk energy ids upward, taking the contiguous run of
    // spots with that id starting where the previous layer ended.
    int nl = 0, start = 0;
    for (int e = 0; e < n_energies; ++e) {
        int end = start;
        while (end < n_spots && spots_out[end].energy_id == e) ++end;
        const int cnt = end - start;
        if (!cnt) continue;
        PbLayer &L = layers_out[nl++];
        L.spot_start = start;
        L.n_spots = cnt;
        L.energy_id = e;
        L.r80 = dvp[(size_t)dvp_len * e + 1];
        L.energy = dvp[(size_t)dvp_len * e];
        L.sx0 = L.sx1 = L.sy0 = L.sy1 = 0.0f;   // culling bounds: see pb_layer_bounds
        L.sh_max = L.mcs_max = 0.0f;
        L.bound_ok = 0;
        start += cnt;
    }
    *n_layers_out = nl;
    return PB_OK;
}

PbStatus pb_spot_geometry(const PbSpot *spots, int n_spots, float vsadx, float vsady,
                          float *geo_out)
{
    if (n_spots < 0 || (n_spots > 0 && (!spots || !geo_out)))
        return set_error(PB_ERR_INVALID, "NULL argument");
    if (!(vsadx != 0.0f) || !(vsady != 0.0f))
        return set_error(PB_ERR_INVALID, "VSADX/VSADY must be non-zero");
    const double ivx = 1.0 / (double)vsadx, ivy = 1.0 / (double)vsady;
    for (int q = 0; q < n_spots; ++q) {
        const double x = spots[q].x, y = spots[q].y;
        const double tx = x * ivx, ty = y * ivy;
        float *o = geo_out + (size_t)PB_SPOT_GEO_FLOATS * q;
        o[0] = (float)x;
        o[1] = (float)y;
        o[2] = (float)(1.0 / (1.0 + tx * tx + ty * ty));
        o[3] = (float)tx;
        o[4] = (float)ty;
        o[5] = (float)(x * y * (ivx - ivy));
        o[6] = 0.0f;
        o[7] = 0.0f;
    }
    return PB_OK;
}

PbStatus pb_rlsp_from_hu(const float *hu_dev, int64_t n, const double *curve_hu,
                         const double *curve_rlsp, int n_curve, float *rlsp_dev, void *stream)
{
    if (n < 0) return set_error(PB_ERR_INVALID, "n must be >= 0");
    if (n > 0 && (!hu_dev || !rlsp_dev)) return set_error(PB_ERR_INVALID, "NULL buffer");
    if (!curve_hu || !curve_rlsp || n_curve < 1 || n_curve > PB_MAX_CURVE)
        return set_error(PB_ERR_INVALID, "curve must have 1..%d points", PB_MAX_CURVE);
    for (int i = 0; i + 1 < n_curve; ++i)
        if (!(curve_hu[i + 1] > curve_hu[i]))
            return set_error(PB_ERR_INVALID, "curve HU values must be strictly increasing");
    return launch_rlsp(hu_dev, n, curve_hu, curve_rlsp, n_curve, rlsp_dev,
                       static_cast<cudaStream_t>(stream));
}

PbStatus pb_texture_create(const float *rlsp_dev, const PbGrid *grid, PbTexture *tex_out,
                           void *stream)
{
    PbStatus s = check_grid(grid);
    if (s != PB_OK) return s;
    if (!rlsp_dev || !tex_out) return set_error(PB_ERR_INVALID, "NULL argument");
    return texture_create(rlsp_dev, *grid, tex_out, static_cast<cudaStream_t>(stream));
}

PbStatus pb_cells_create(const float *rlsp_dev, const PbGrid *grid, PbTexture *cells_out,
                         void *stream)
{
    PbStatus s = check_grid(grid);
    if (s != PB_OK) return s;
    if (!rlsp_dev || !cells_out) return set_error(PB_ERR_INVALID, "NULL argument");
    return texture_create(rlsp_dev, *grid, cells_out, static_cast<cudaStream_t>(stream), false);
}

PbStatus pb_texture_update(PbTexture tex, const float *rlsp_dev, void *stream)
{
    if (!tex || !rlsp_dev) return set_error(PB_ERR_INVALID, "NULL argument");
    return texture_update(tex, rlsp_dev, static_cast<cudaStream_t>(stream));
}

PbStatus pb_texture_destroy(PbTexture tex)
{
    texture_destroy(tex);
    return PB_OK;
}

PbStatus pb_wet(const float *rlsp_dev, PbTexture tex, const PbGrid *grid,
                const PbBeamGeom *beams, int n_beams, float *raw_work_dev, float *wet_dev,
                int *status_dev, void *stream)
{
    PbStatus s = check_wet_args(rlsp_dev, tex, grid, beams, n_beams, wet_dev);
    if (s != PB_OK) return s;
    if (!raw_work_dev) return set_error(PB_ERR_INVALID, "NULL argument");
    return launch_wet(rlsp_dev, texture_object(tex), texture_cells(tex), *grid, beams, n_beams,
                      raw_work_dev, wet_dev, status_dev, static_cast<cudaStream_t>(stream));
}

PbStatus pb_smooth_dirs(float *cos_out, float *sin_out)
{
    if (!cos_out || !sin_out) return set_error(PB_ERR_INVALID, "NULL argument");
    return device_smooth_dirs(cos_out, sin_out);
}

PbStatus pb_smooth_table(const PbGrid *grid, const PbBeamGeom *beams, int n_beams, int beam,
                         int *off, float *hh, unsigned *tmask, int *margin)
{
    PbStatus s = check_grid(grid);
    if (s != PB_OK) return s;
    if (!beams || !off || !hh || !tmask || !margin)
        return set_error(PB_ERR_INVALID, "NULL argument");
    if (n_beams <= 0 || n_beams > PB_MAX_BEAMS)
        return set_error(PB_ERR_INVALID, "n_beams must be in [1, %d] (got %d)", PB_MAX_BEAMS,
                         n_beams);
    if (beam < 0 || beam >= n_beams)
        return set_error(PB_ERR_INVALID, "beam %d is not in [0, %d)", beam, n_beams);
    smooth_table_host(*grid, beams, n_beams, beam, off, hh, tmask, margin);
    return PB_OK;
}

PbStatus pb_dose(const PbGrid *grid, const PbBeam *beams, int n_beams, const float *wet_dev,
                 const PbLayer *layers_dev, const float *spot_geo_dev, const float *mu_dev,
                 float scale, float *dose_dev, float *beam_dose_dev, void *stream)
{
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!dose_dev) return set_error(PB_ERR_INVALID, "dose is NULL");
    if (!mu_dev) {
        for (int b = 0; b < n_beams; ++b)
            if (beams[b].n_layers) return set_error(PB_ERR_INVALID, "mu is NULL");
    }
    return launch_dose(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev, mu_dev, scale,
                       dose_dev, beam_dose_dev, static_cast<cudaStream_t>(stream));
}

long long pb_tile_order_count(const PbGrid *grid)
{
    return check_grid(grid) == PB_OK ? tile_order_count(*grid) : -1;
}

PbStatus pb_tile_order_tile(int *tile_voxels)
{
    if (!tile_voxels) return set_error(PB_ERR_INVALID, "tile_voxels is NULL");
    tile_order_tile(tile_voxels);
    return PB_OK;
}

size_t pb_tile_order_work_size(const PbGrid *grid)
{
    return check_grid(grid) == PB_OK ? tile_order_work_size(*grid) : 0;
}

PbStatus pb_tile_order(const PbGrid *grid, const PbBeam *beams, int n_beams,
                       const float *wet_dev, const PbLayer *layers_dev, void *work_dev,
                       int *order_dev, void *stream)
{
    // the order reads the layers and the model tables, not the spots
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, nullptr, false);
    if (s != PB_OK) return s;
    if (!work_dev || !order_dev) return set_error(PB_ERR_INVALID, "work or order is NULL");
    return launch_tile_order(*grid, beams, n_beams, wet_dev, layers_dev, work_dev, order_dev,
                             static_cast<cudaStream_t>(stream));
}

PbStatus pb_dose_ordered(const PbGrid *grid, const PbBeam *beams, int n_beams,
                         const float *wet_dev, const PbLayer *layers_dev,
                         const float *spot_geo_dev, const float *mu_dev, float scale,
                         float *dose_dev, float *beam_dose_dev, const int *order_dev,
                         void *stream)
{
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!dose_dev) return set_error(PB_ERR_INVALID, "dose is NULL");
    if (!mu_dev) {
        for (int b = 0; b < n_beams; ++b)
            if (beams[b].n_layers) return set_error(PB_ERR_INVALID, "mu is NULL");
    }
    return launch_dose(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev, mu_dev, scale,
                       dose_dev, beam_dose_dev, static_cast<cudaStream_t>(stream), -1,
                       order_dev);
}

PbStatus pb_dose_adjoint_ordered(const PbGrid *grid, const PbBeam *beams, int n_beams,
                                 const float *wet_dev, const PbLayer *layers_dev,
                                 const float *spot_geo_dev, const float *dobj_dose_dev,
                                 float scale, float *grad_dev, const int *order_dev,
                                 void *stream)
{
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!dobj_dose_dev || !grad_dev) return set_error(PB_ERR_INVALID, "NULL argument");
    return launch_adjoint(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev,
                          dobj_dose_dev, scale, grad_dev, static_cast<cudaStream_t>(stream), -1,
                          order_dev);
}

PbStatus pb_dose_adjoint(const PbGrid *grid, const PbBeam *beams, int n_beams,
                         const float *wet_dev, const PbLayer *layers_dev,
                         const float *spot_geo_dev, const float *dobj_dose_dev, float scale,
                         float *grad_dev, void *stream)
{
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!dobj_dose_dev || !grad_dev) return set_error(PB_ERR_INVALID, "NULL argument");
    return launch_adjoint(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev,
                          dobj_dose_dev, scale, grad_dev, static_cast<cudaStream_t>(stream));
}

PbStatus pb_dose_adjoint_variant(const PbGrid *grid, const PbBeam *beams, int n_beams,
                                 const float *wet_dev, const PbLayer *layers_dev,
                                 const float *spot_geo_dev, const float *dobj_dose_dev,
                                 float scale, float *grad_dev, int variant, void *stream)
{
    if (variant < 0 || variant >= dose_variant_count())
        return set_error(PB_ERR_INVALID, "variant must be in [0, %d)", dose_variant_count());
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!dobj_dose_dev || !grad_dev) return set_error(PB_ERR_INVALID, "NULL argument");
    return launch_adjoint(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev,
                          dobj_dose_dev, scale, grad_dev, static_cast<cudaStream_t>(stream),
                          variant);
}

size_t pb_objective_work_size(void) { return objective_work_size(); }

PbStatus pb_objective(const float *dose_dev, const float *presc_dev, const float *weight_dev,
                      int64_t n, double *obj_dev, float *resid_dev, void *work_dev,
                      void *stream)
{
    if (n < 0) return set_error(PB_ERR_INVALID, "n must be >= 0");
    if (!dose_dev || !presc_dev || !weight_dev || !obj_dev || !work_dev)
        return set_error(PB_ERR_INVALID, "NULL argument");
    return launch_objective(dose_dev, presc_dev, weight_dev, n, obj_dev, resid_dev, work_dev,
                            static_cast<cudaStream_t>(stream));
}

PbStatus pb_count_pairs(const PbGrid *grid, const PbBeam *beams, int n_beams,
                        const float *wet_dev, const PbLayer *layers_dev,
                        unsigned long long *count_dev, void *stream)
{
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev,
                             reinterpret_cast<const float *>(1));
    if (s != PB_OK) return s;
    if (!count_dev) return set_error(PB_ERR_INVALID, "count is NULL");
    return launch_count_pairs(*grid, beams, n_beams, wet_dev, layers_dev, count_dev,
                              static_cast<cudaStream_t>(stream));
}

PbStatus pb_dose_adjoint_positions(const PbGrid *grid, const PbBeam *beams, int n_beams,
                                   const float *wet_dev, const PbLayer *layers_dev,
                                   const float *spot_geo_dev, const float *mu_dev,
                                   const float *dobj_dose_dev, float scale, float *grad_dev,
                                   float *grad_x_dev, float *grad_y_dev, void *stream)
{
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!dobj_dose_dev || !grad_x_dev || !grad_y_dev)
        return set_error(PB_ERR_INVALID, "NULL argument");
    for (int b = 0; b < n_beams; ++b)
        if (beams[b].n_layers && !mu_dev) return set_error(PB_ERR_INVALID, "mu is NULL");
    return launch_adjoint_positions(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev,
                                    mu_dev, dobj_dose_dev, scale, grad_dev, grad_x_dev,
                                    grad_y_dev, static_cast<cudaStream_t>(stream));
}

PbStatus pb_count_evaluated(const PbGrid *grid, const PbBeam *beams, int n_beams,
                            const float *wet_dev, const PbLayer *layers_dev,
                            const float *spot_geo_dev, unsigned long long *count_dev,
                            void *stream)
{
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!count_dev) return set_error(PB_ERR_INVALID, "count is NULL");
    return launch_count_evaluated(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev,
                                  count_dev, static_cast<cudaStream_t>(stream));
}

PbStatus pb_count_evaluated_adjoint(const PbGrid *grid, const PbBeam *beams, int n_beams,
                                    const float *wet_dev, const PbLayer *layers_dev,
                                    const float *spot_geo_dev, const float *dobj_dose_dev,
                                    float scale, unsigned long long *count_dev, void *stream)
{
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!dobj_dose_dev || !count_dev) return set_error(PB_ERR_INVALID, "NULL argument");
    return launch_count_evaluated(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev,
                                  count_dev, static_cast<cudaStream_t>(stream), -1,
                                  dobj_dose_dev, scale);
}

PbStatus pb_host_register(void *host_ptr, size_t bytes)
{
    if (!host_ptr || bytes == 0) return set_error(PB_ERR_INVALID, "NULL or empty host range");
    const cudaError_t e = cudaHostRegister(host_ptr, bytes, cudaHostRegisterDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();   // leave no error behind for the next launch check
        return set_error(PB_ERR_CUDA, "cudaHostRegister: %s", cudaGetErrorString(e));
    }
    return PB_OK;
}

PbStatus pb_host_unregister(void *host_ptr)
{
    if (!host_ptr) return set_error(PB_ERR_INVALID, "NULL host pointer");
    const cudaError_t e = cudaHostUnregister(host_ptr);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(PB_ERR_CUDA, "cudaHostUnregister: %s", cudaGetErrorString(e));
    }
    return PB_OK;
}

PbStatus pb_measure_ex2_rate(double *ops_per_s, void *stream)
{
    if (!ops_per_s) return set_error(PB_ERR_INVALID, "ops_per_s is NULL");
    return measure_ex2_rate(ops_per_s, static_cast<cudaStream_t>(stream));
}

PbStatus pb_layer_bounds(const PbBeam *beams, int n_beams, PbLayer *layers_dev,
                         const float *spot_geo_dev, void *stream)
{
    if (!beams || n_beams <= 0 || n_beams > PB_MAX_BEAMS)
        return set_error(PB_ERR_INVALID, "n_beams must be in [1, %d] (got %d)", PB_MAX_BEAMS,
                         n_beams);
    for (int b = 0; b < n_beams; ++b) {
        const PbBeam &B = beams[b];
        if (B.n_layers < 0 || B.layer_start < 0 || B.spot_start < 0 || B.n_spots < 0)
            return set_error(PB_ERR_INVALID, "beam %d: negative layer/spot range", b);
        if (B.n_layers == 0) continue;
        if (!layers_dev || !spot_geo_dev)
            return set_error(PB_ERR_INVALID, "layers/spot geometry is NULL");
        if (!B.sigmas_dev) return set_error(PB_ERR_INVALID, "beam %d: model table is NULL", b);
        if (B.lut_len <= 0 || B.lut_len > PB_MAX_LUT_LEN)
            return set_error(PB_ERR_INVALID, "beam %d: lut_len must be in [1, %d] (got %d)", b,
                             PB_MAX_LUT_LEN, B.lut_len);
    }
    return launch_layer_bounds(beams, n_beams, layers_dev, spot_geo_dev,
                               static_cast<cudaStream_t>(stream));
}

}  // extern "C"

// ------------------------------------------------------- host drop-in level

namespace pb {

struct DevBuf {
    void *p = nullptr;
    size_t cap = 0;
};

enum { kBufRlsp, kBufRaw, kBufWet, kBufDose, kBufLayers, kBufGeo, kBufMu, kBufDvp,
       kBufDep, kBufSig, kBufIdd, kBufStatus, kBufOrderWork, kBufOrder, kBufCount };

struct DevState {
    std::mutex m;
    DevBuf buf[kBufCount];
    uint64_t tex = 0;   // RLSP texture of the last raytrace call's grid
};

constexpr int kMaxDevices = 64;
static DevState g_dev[kMaxDevices];

static PbStatus ensure(DevBuf &b, size_t bytes)
{
    if (bytes == 0) bytes = 16;
    if (b.cap >= bytes) return PB_OK;
    if (b.p) {
        cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
    }
    PbStatus s = check_cuda(cudaMalloc(&b.p, bytes), "cudaMalloc");
    if (s != PB_OK) return s;
    b.cap = bytes;
    return PB_OK;
}

static PbStatus select_device(int gpu_id)
{
    int n = 0;
    PbStatus s = check_cuda(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
    if (s != PB_OK) return s;
    if (gpu_id < 0 || gpu_id >= n || gpu_id >= kMaxDevices)
        return set_error(PB_ERR_CUDA, "invalid device ordinal %d (%d devices)", gpu_id, n);
    return check_cuda(cudaSetDevice(gpu_id), "cudaSetDevice");
}

static PbStatus grid_from_dims(const int64_t dims[3], float spacing, PbGrid &g)
{
    if (!dims) return set_error(PB_ERR_INVALID, "dims is NULL");
    if (dims[0] <= 0 || dims[1] <= 0 || dims[2] <= 0 || dims[0] > INT32_MAX ||
        dims[1] > INT32_MAX || dims[2] > INT32_MAX)
        return set_error(PB_ERR_INVALID, "volume dimensions must be positive");
    g.nz = (int)dims[0];
    g.ny = (int)dims[1];
    g.nx = (int)dims[2];
    g.spacing = spacing;
    return check_grid(&g);
}

#define PB_TRY(expr)                   \
    do {                               \
        PbStatus _s = (expr);          \
        if (_s != PB_OK) return _s;    \
    } while (0)

}  // namespace pb

extern "C" {

PbStatus pb_proton_raytrace_host(int gpu_id, double vsadx, double vsady, const float *rlsp,
                                 const int64_t dims[3], float spacing, const float origin[3],
                                 const float iso[3], double gantry_deg, double couch_deg,
                                 float *wet_out)
{
    if (!rlsp || !origin || !iso || !wet_out) return set_error(PB_ERR_INVALID, "NULL argument");
    PbGrid g;
    PB_TRY(grid_from_dims(dims, spacing, g));
    PB_TRY(select_device(gpu_id));
    PbBeamGeom bg;
    PB_TRY(pb_beam_setup(gantry_deg, couch_deg, vsadx, vsady, iso, origin, &bg));
    DevState &D = g_dev[gpu_id];
    std::lock_guard<std::mutex> lock(D.m);
    const size_t vb = sizeof(float) * (size_t)g.nx * g.ny * g.nz;
    PB_TRY(ensure(D.buf[kBufRlsp], vb));
    PB_TRY(ensure(D.buf[kBufRaw], vb));
    PB_TRY(ensure(D.buf[kBufWet], vb));
    PB_TRY(ensure(D.buf[kBufStatus], sizeof(int)));
    float *d_rlsp = static_cast<float *>(D.buf[kBufRlsp].p);
    float *d_raw = static_cast<float *>(D.buf[kBufRaw].p);
    float *d_wet = static_cast<float *>(D.buf[kBufWet].p);
    int *d_status = static_cast<int *>(D.buf[kBufStatus].p);
    cudaStream_t st = 0;
    PB_TRY(check_cuda(cudaMemcpyAsync(d_rlsp, rlsp, vb, cudaMemcpyHostToDevice, st), "H2D rlsp"));
    PB_TRY(check_cuda(cudaMemsetAsync(d_status, 0, sizeof(int), st), "memset status"));
    if (D.tex && !texture_matches(D.tex, g)) {
        PB_TRY(check_cuda(cudaStreamSynchronize(st), "synchronize"));
        texture_destroy(D.tex);
        D.tex = 0;
    }
    if (D.tex)
        PB_TRY(texture_update(D.tex, d_rlsp, st));
    else
        PB_TRY(texture_create(d_rlsp, g, &D.tex, st));
    PB_TRY(launch_wet(d_rlsp, texture_object(D.tex), texture_cells(D.tex), g, &bg, 1, d_raw, d_wet, d_status, st));
    int status = 0;
    PB_TRY(check_cuda(cudaMemcpyAsync(wet_out, d_wet, vb, cudaMemcpyDeviceToHost, st), "D2H wet"));
    PB_TRY(check_cuda(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st),
                      "D2H status"));
    PB_TRY(check_cuda(cudaStreamSynchronize(st), "synchronize"));
    if (status & PB_ERR_RAY_CAP)
        return set_error(PB_ERR_RAY_CAP, "a WET ray reached its step cap");
    return PB_OK;
}

PbStatus pb_proton_spot_host(int gpu_id, double vsadx, double vsady, const float *dvp,
                             const float *depths, const float *sigmas, const float *idds,
                             int n_energies, int lut_len, int dvp_len, const float *wet,
                             const int64_t dims[3], float spacing, const float origin[3],
                             const float iso[3], double gantry_deg, double couch_deg,
                             const float *spot_list, int n_spots, float *dose_out)
{
    if (!dvp || !depths || !sigmas || !idds || !wet || !origin || !iso || !dose_out ||
        (n_spots > 0 && !spot_list))
        return set_error(PB_ERR_INVALID, "NULL argument");
    if (n_energies <= 0 || lut_len <= 0 || lut_len > PB_MAX_LUT_LEN || dvp_len < 5 ||
        n_spots < 0)
        return set_error(PB_ERR_INVALID, "invalid model table shape");
    PbGrid g;
    PB_TRY(grid_from_dims(dims, spacing, g));
    PB_TRY(select_device(gpu_id));
    PbBeamGeom bg;
    PB_TRY(pb_beam_setup(gantry_deg, couch_deg, vsadx, vsady, iso, origin, &bg));

    std::vector<PbSpot> spots((size_t)n_spots);
    std::vector<PbLayer> layers((size_t)n_energies);
    int n_layers = 0;
    PB_TRY(pb_build_layers(spot_list, n_spots, dvp, dvp_len, n_energies, spots.data(),
                           layers.data(), &n_layers, nullptr));
    std::vector<float> geo((size_t)PB_SPOT_GEO_FLOATS * n_spots);
    std::vector<float> mu((size_t)n_spots);
    PB_TRY(pb_spot_geometry(spots.data(), n_spots, bg.vsadx, bg.vsady, geo.data()));
    for (int q = 0; q < n_spots; ++q) mu[q] = spots[q].mu;

    DevState &D = g_dev[gpu_id];
    std::lock_guard<std::mutex> lock(D.m);
    const size_t vb = sizeof(float) * (size_t)g.nx * g.ny * g.nz;
    const size_t tb = sizeof(float) * (size_t)n_energies * lut_len;
    PB_TRY(ensure(D.buf[kBufWet], vb));
    PB_TRY(ensure(D.buf[kBufDose], vb));
    PB_TRY(ensure(D.buf[kBufLayers], sizeof(PbLayer) * layers.size()));
    PB_TRY(ensure(D.buf[kBufGeo], sizeof(float) * geo.size()));
    PB_TRY(ensure(D.buf[kBufMu], sizeof(float) * mu.size()));
    PB_TRY(ensure(D.buf[kBufDvp], sizeof(float) * (size_t)n_energies * dvp_len));
    PB_TRY(ensure(D.buf[kBufDep], tb));
    PB_TRY(ensure(D.buf[kBufSig], tb));
    PB_TRY(ensure(D.buf[kBufIdd], tb));
    PB_TRY(ensure(D.buf[kBufOrderWork], tile_order_work_size(g)));
    PB_TRY(ensure(D.buf[kBufOrder], sizeof(int) * (size_t)tile_order_count(g)));
    cudaStream_t st = 0;
    auto h2d = [&](int slot, const void *src, size_t bytes) -> PbStatus {
        if (!bytes) return PB_OK;
        return check_cuda(cudaMemcpyAsync(D.buf[slot].p, src, bytes, cudaMemcpyHostToDevice, st),
                          "H2D");
    };
    float *d_dose = static_cast<float *>(D.buf[kBufDose].p);
    if (n_layers == 0) {
        // No layer holds a spot: the reference launches an empty grid and
        // returns its zeroed dose buffer.
        PB_TRY(check_cuda(cudaMemsetAsync(d_dose, 0, vb, st), "memset dose"));
    } else {
        PB_TRY(h2d(kBufWet, wet, vb));
        PB_TRY(h2d(kBufLayers, layers.data(), sizeof(PbLayer) * (size_t)n_layers));
        PB_TRY(h2d(kBufGeo, geo.data(), sizeof(float) * geo.size()));
        PB_TRY(h2d(kBufMu, mu.data(), sizeof(float) * mu.size()));
        PB_TRY(h2d(kBufDvp, dvp, sizeof(float) * (size_t)n_energies * dvp_len));
        PB_TRY(h2d(kBufDep, depths, tb));
        PB_TRY(h2d(kBufSig, sigmas, tb));
        PB_TRY(h2d(kBufIdd, idds, tb));
        PbBeam B;
        B.geom = bg;
        B.layer_start = 0;
        B.n_layers = n_layers;
        B.spot_start = 0;
        B.n_spots = n_spots;
        B.dvp_dev = static_cast<const float *>(D.buf[kBufDvp].p);
        B.depths_dev = static_cast<const float *>(D.buf[kBufDep].p);
        B.sigmas_dev = static_cast<const float *>(D.buf[kBufSig].p);
        B.idds_dev = static_cast<const float *>(D.buf[kBufIdd].p);
        B.n_energies = n_energies;
        B.lut_len = lut_len;
        B.dvp_len = dvp_len;
        PB_TRY(launch_layer_bounds(&B, 1, static_cast<PbLayer *>(D.buf[kBufLayers].p),
                                   static_cast<const float *>(D.buf[kBufGeo].p), st));
        // the tiles in the order of their estimated work (pb_tile_order)
        PB_TRY(launch_tile_order(g, &B, 1, static_cast<const float *>(D.buf[kBufWet].p),
                                 static_cast<const PbLayer *>(D.buf[kBufLayers].p),
                                 D.buf[kBufOrderWork].p, static_cast<int *>(D.buf[kBufOrder].p),
                                 st));
        PB_TRY(launch_dose(g, &B, 1, static_cast<const float *>(D.buf[kBufWet].p),
                           static_cast<const PbLayer *>(D.buf[kBufLayers].p),
                           static_cast<const float *>(D.buf[kBufGeo].p),
                           static_cast<const float *>(D.buf[kBufMu].p), 1.0f, d_dose, nullptr,
                           st, -1, static_cast<const int *>(D.buf[kBufOrder].p)));
    }
    PB_TRY(check_cuda(cudaMemcpyAsync(dose_out, d_dose, vb, cudaMemcpyDeviceToHost, st),
                      "D2H dose"));
    return check_cuda(cudaStreamSynchronize(st), "synchronize");
}

}  // extern "C"

// ------------------------------------------------------------ variants, batch

namespace pb {

// work_dev layout: [queue counter | padding to 256 B][WET records][dose records]
static size_t batch_wet_offset() { return 256; }
static size_t batch_dose_offset(int n_plans)
{
    const size_t w = batch_wet_offset() + batch_wet_size() * (size_t)n_plans * PB_MAX_BEAMS;
    return (w + 255) & ~(size_t)255;
}

}  // namespace pb

extern "C" {

int pb_dose_variant_count(void) { return dose_variant_count(); }

int pb_dose_variant_default(void) { return dose_variant_default(); }

const char *pb_dose_variant_name(int variant) { return dose_variant_name(variant); }

PbStatus pb_dose_variant(const PbGrid *grid, const PbBeam *beams, int n_beams,
                         const float *wet_dev, const PbLayer *layers_dev,
                         const float *spot_geo_dev, const float *mu_dev, float scale,
                         float *dose_dev, int variant, void *stream)
{
    if (variant < 0 || variant >= dose_variant_count())
        return set_error(PB_ERR_INVALID, "variant must be in [0, %d)", dose_variant_count());
    PbStatus s = check_beams(grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev);
    if (s != PB_OK) return s;
    if (!dose_dev || !mu_dev) return set_error(PB_ERR_INVALID, "NULL argument");
    return launch_dose(*grid, beams, n_beams, wet_dev, layers_dev, spot_geo_dev, mu_dev, scale,
                       dose_dev, nullptr, static_cast<cudaStream_t>(stream), variant);
}

size_t pb_batch_work_size(int n_plans)
{
    if (n_plans <= 0) return 0;
    return batch_dose_offset(n_plans) + batch_dose_size() * (size_t)n_plans;
}

PbStatus pb_batch_setup(const PbBatchPlan *plans, int n_plans, void *work_dev,
                        PbBatchInfo *info, void *stream)
{
    if (!plans || n_plans <= 0 || !work_dev || !info)
        return set_error(PB_ERR_INVALID, "NULL argument or empty batch");
    for (int p = 0; p < n_plans; ++p) {
        const PbBatchPlan &P = plans[p];
        PbStatus s = check_beams(&P.grid, P.beams, P.n_beams, P.wet_dev, P.layers_dev,
                                 P.spot_geo_dev);
        if (s != PB_OK)
            return set_error(s, "plan %d: %s", p, pb_last_error());
        if ((!P.rlsp_dev && !texture_samples(P.tex)) || !P.raw_work_dev || !P.dose_dev ||
            !P.mu_dev)
            return set_error(PB_ERR_INVALID, "plan %d: NULL buffer", p);
        if (P.tex && !texture_matches(P.tex, P.grid))
            return set_error(PB_ERR_INVALID, "plan %d: texture extent differs from the grid", p);
    }
    // WET records in plan order
    std::vector<unsigned char> wet_items(batch_wet_size() * (size_t)n_plans * PB_MAX_BEAMS);
    long long bricks = 0;
    int n_wet = 0;
    for (int p = 0; p < n_plans; ++p) {
        const PbBatchPlan &P = plans[p];
        PbBeamGeom geoms[PB_MAX_BEAMS];
        for (int b = 0; b < P.n_beams; ++b) geoms[b] = P.beams[b].geom;
        bricks += fill_batch_wet(wet_items.data(), n_wet, P.grid, geoms, P.n_beams, P.rlsp_dev,
                                 texture_object(P.tex), texture_cells(P.tex), P.raw_work_dev,
                                 P.wet_dev, bricks);
        n_wet += P.n_beams;
    }
    // dose records, most expensive tiles first (spots over all beams)
    std::vector<int> order((size_t)n_plans);
    std::vector<long long> cost((size_t)n_plans);
    for (int p = 0; p < n_plans; ++p) {
        order[p] = p;
        long long c = 0;
        for (int b = 0; b < plans[p].n_beams; ++b) c += plans[p].beams[b].n_spots;
        cost[p] = c;
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return cost[a] > cost[b]; });
    std::vector<unsigned char> dose_items(batch_dose_size() * (size_t)n_plans);
    long long tiles = 0;
    for (int q = 0; q < n_plans; ++q) {
        const PbBatchPlan &P = plans[order[q]];
        BatchDose &D = *reinterpret_cast<BatchDose *>(dose_items.data() + batch_dose_size() * q);
        fill_batch_dose(D, P.grid, P.beams, P.n_beams, P.scale, P.wet_dev, P.layers_dev,
                        P.spot_geo_dev, P.mu_dev, P.dose_dev, tiles);
        tiles += plan_tiles(P.grid);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char *w = static_cast<unsigned char *>(work_dev);
    PbStatus s = check_cuda(cudaMemcpyAsync(w + batch_wet_offset(), wet_items.data(),
                                            batch_wet_size() * (size_t)n_wet,
                                            cudaMemcpyHostToDevice, st), "H2D batch WET records");
    if (s != PB_OK) return s;
    s = check_cuda(cudaMemcpyAsync(w + batch_dose_offset(n_plans), dose_items.data(),
                                   dose_items.size(), cudaMemcpyHostToDevice, st),
                   "H2D batch dose records");
    if (s != PB_OK) return s;
    s = check_cuda(cudaStreamSynchronize(st), "synchronize");
    if (s != PB_OK) return s;
    info->n_bricks = bricks;
    info->n_tiles = tiles;
    info->n_wet_items = n_wet;
    info->n_plans = n_plans;
    return PB_OK;
}

PbStatus pb_batch_run(const PbBatchInfo *info, void *work_dev, int flags, int variant,
                      int blocks_per_sm, int *status_dev, void *stream)
{
    if (!info || !work_dev || info->n_plans <= 0)
        return set_error(PB_ERR_INVALID, "NULL argument or empty batch");
    if (variant < 0 || variant >= dose_variant_count())
        return set_error(PB_ERR_INVALID, "variant must be in [0, %d)", dose_variant_count());
    if (blocks_per_sm <= 0 || blocks_per_sm > 32)
        return set_error(PB_ERR_INVALID, "blocks_per_sm must be in [1, 32]");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char *w = static_cast<unsigned char *>(work_dev);
    if (flags & PB_BATCH_WET) {
        PbStatus s = launch_wet_batch(w + batch_wet_offset(), info->n_wet_items, info->n_bricks,
                                      status_dev, st);
        if (s != PB_OK) return s;
    }
    if (flags & PB_BATCH_DOSE) {
        int dev = 0, sms = 0;
        PbStatus s = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
        if (s != PB_OK) return s;
        s = check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                       "cudaDeviceGetAttribute");
        if (s != PB_OK) return s;
        return launch_dose_batch(w + batch_dose_offset(info->n_plans), info->n_plans,
                                 info->n_tiles, reinterpret_cast<unsigned long long *>(w), variant,
                                 blocks_per_sm * sms, st);
    }
    return PB_OK;
}

}  // extern "C"
