/*
 * pb_b200.h -- C ABI of the B200 proton pencil-beam dose library
 * (libpb_b200.so).
 *
 * Replaces the native half of DoseCUDA's proton path:
 *   DoseCUDA/dose_kernels/IMPTClasses.cuh:90-91
 *       void proton_raytrace_cuda(int gpu_id, CudaDose*, CudaBeam*);
 *       void proton_spot_cuda(int gpu_id, IMPTDose*, IMPTBeam*);
 *   and the CPython wrappers that feed them,
 *   DoseCUDA/dose_kernels/dosemodule.cu:104-201 (proton_raytrace) and
 *   dosemodule.cu:243-374 (proton_spot).
 *
 * Conventions
 *   - Plain C types only.  Every function returns a PbStatus; none throws.
 *     pb_last_error() gives the text of the last failure on this thread.
 *   - Volumes are C-ordered (nz, ny, nx) float32, x fastest; the linear
 *     index of voxel (i, j, k) is i + nx*(j + ny*k)  (CudaClasses.cuh:96-98).
 *   - Functions whose pointer arguments are named *_dev take device
 *     pointers on the current CUDA device and are ordered on `stream`
 *     (a cudaStream_t passed as void*; NULL = legacy default stream).  They
 *     allocate nothing: buffers, including work space, come from the caller.
 *   - Functions named *_host take host pointers, select `gpu_id`, and
 *     return when the result is in host memory (the reference's contract).
 *     They keep grow-only device buffers per device between calls.
 *   - WET is in cm, distances in mm, angles in degrees, dose in the IDD
 *     table's units per mm^2 per MU (IMPTClasses.cu:243-244).
 */
#ifndef PB_B200_H
#define PB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    PB_OK = 0,
    PB_ERR_INVALID = 1,      /* bad argument (null pointer, size, shape)   */
    PB_ERR_CUDA = 2,         /* a CUDA runtime call or launch failed       */
    PB_ERR_NOMEM = 3,        /* host or device allocation failed           */
    PB_ERR_RAY_CAP = 4,      /* a WET ray reached its step cap             */
    PB_ERR_UNSUPPORTED = 5   /* valid request this build cannot serve      */
} PbStatus;

#define PB_MAX_BEAMS 16      /* beams per plan in one launch               */
#define PB_MAX_LUT_LEN 512   /* LUT rows per energy (reference: 400)       */
#define PB_MAX_CURVE 64      /* points of an HU -> RLSP curve              */

/* Voxel grid: isotropic spacing only (dosemodule.cu:146, plan_impt.py:177). */
typedef struct {
    int nx, ny, nz;
    float spacing;           /* mm */
} PbGrid;

/* Beam geometry after the reference's set-up: gantry' = fmod(g+180, 360),
 * iso' = iso - origin, source at (vsadx+vsady)/2 rotated by gantry' about z
 * and couch about y (CudaClasses.cu:17-51, dosemodule.cu:148-175). */
typedef struct {
    float iso[3];            /* isocentre minus grid origin, mm            */
    float src[3];            /* source relative to the isocentre, mm       */
    float singa, cosga;      /* gantry' sine / cosine                      */
    float sinta, costa;      /* couch sine / cosine                        */
    float vsadx, vsady;      /* virtual source-axis distances, mm          */
} PbBeamGeom;

/* A spot as the reference stores it (IMPTClasses.cuh:8-15). */
typedef struct {
    float x, y, mu;
    int energy_id;
} PbSpot;

/* An energy layer (IMPTClasses.cuh:17-26); spot_start is relative to the
 * beam's first spot.  The fields after `energy` have no counterpart in the
 * reference: bounds that let the dose kernels skip a layer for a whole
 * voxel tile without evaluating it (pb_layer_bounds fills them on the
 * device; pb_build_layers leaves bound_ok = 0, which disables the test). */
typedef struct {
    int spot_start, n_spots, energy_id;
    float r80, energy;
    float sx0, sx1, sy0, sy1;    /* box of the spots' (x, y) at the isocentre */
    float sh_max;                /* >= the nuclear-halo sigma at any depth, mm */
    float mcs_max;               /* >= |sigma_mcs| of the layer's LUT row, mm  */
    int bound_ok;                /* 1 when the four lines above are filled    */
} PbLayer;

/* One beam of a plan as the dose kernels see it.  Model tables are device
 * pointers: dvp is n_energies x dvp_len (energy, R80, A, B, C), the LUTs are
 * n_energies x lut_len (plan_impt.py:63-149). */
typedef struct {
    PbBeamGeom geom;
    int layer_start, n_layers;   /* into the plan's layer array            */
    int spot_start, n_spots;     /* into the plan's spot arrays            */
    const float *dvp_dev;
    const float *depths_dev, *sigmas_dev, *idds_dev;
    int n_energies, lut_len, dvp_len;
} PbBeam;

/* Number of floats of per-spot geometry that pb_spot_geometry writes. */
#define PB_SPOT_GEO_FLOATS 8

/* ---------------------------------------------------------------- host */

/* Text of the last error on this thread ("" if none). */
const char *pb_last_error(void);

/* Library version string. */
const char *pb_version(void);

/* Beam set-up, as dosemodule.cu:148-175 + CudaClasses.cu:17-51 do it. */
PbStatus pb_beam_setup(double gantry_deg, double couch_deg, double vsadx,
                       double vsady, const float iso[3], const float origin[3],
                       PbBeamGeom *out);

/* Sort spots by energy id (ties keep input order) and group them into
 * layers like importLayers (dosemodule.cu:204-225, IMPTClasses.cu:29-67).
 * spot_list is n_spots x 4 float (x, y, mu, energy_id); the energy id is
 * truncated to int.  dvp is host n_energies x dvp_len.  layers_out needs
 * room for n_energies entries; perm_out (nullable) receives, for each
 * sorted spot, its row in spot_list. */
PbStatus pb_build_layers(const float *spot_list, int n_spots, const float *dvp,
                         int dvp_len, int n_energies, PbSpot *spots_out,
                         PbLayer *layers_out, int *n_layers_out, int *perm_out);

/* Per-spot geometry for the dose kernels: PB_SPOT_GEO_FLOATS floats per
 * spot (x, y, 1/|t|^2, x/VSADX, y/VSADY, x*y*(1/VSADX-1/VSADY), 0, 0) with
 * t = (x/VSADX, y/VSADY, -1); the first four (16 bytes) are all that the
 * per-tile spot cull reads. */
PbStatus pb_spot_geometry(const PbSpot *spots, int n_spots, float vsadx,
                          float vsady, float *geo_out);

/* -------------------------------------------------------------- device */

/* HU -> RLSP with numpy.interp semantics in FP64, rounded to FP32
 * (plan_impt.py:158-168).  The curve is host data, increasing in HU. */
PbStatus pb_rlsp_from_hu(const float *hu_dev, int64_t n, const double *curve_hu,
                         const double *curve_rlsp, int n_curve, float *rlsp_dev,
                         void *stream);

/* Handle of a 3-D texture holding an RLSP volume with the reference's
 * sampling state: float channel, linear filter, border 0, unnormalised
 * coordinates (TextureClasses.cu:14-41, IMPTClasses.cu:292).  The texture
 * unit's filter weights are fixed point, so samples through it differ
 * slightly from exact trilinear interpolation; the reference's WET is
 * defined by them.  Creating one allocates a CUDA array.  The handle also
 * holds per-cell records (whether each 2x2x2 block of texels is flat, and
 * how far the nearest non-flat one is) from which pb_wet adds whole runs of
 * samples through flat regions at once. */
typedef uint64_t PbTexture;

PbStatus pb_texture_create(const float *rlsp_dev, const PbGrid *grid,
                           PbTexture *tex_out, void *stream);
/* A handle with the cell records only (no texture, no CUDA array), for
 * exact-trilinear WET with the same runs through flat regions.  No
 * counterpart in the reference. */
PbStatus pb_cells_create(const float *rlsp_dev, const PbGrid *grid, PbTexture *cells_out,
                         void *stream);
/* Refill an existing handle (either kind) from a volume of the same grid. */
PbStatus pb_texture_update(PbTexture tex, const float *rlsp_dev, void *stream);
PbStatus pb_texture_destroy(PbTexture tex);

/* WET (cm) of every voxel for n_beams beams: the ray trace toward the
 * source (CudaClasses.cu:180-228, accumulated in FP64) followed by the
 * lateral smoothing (IMPTClasses.cu:139-202).
 *   tex from pb_texture_create: RLSP is sampled through the texture (the
 *             reference's samples); rlsp_dev is not read and may be NULL.
 *   tex from pb_cells_create, or 0: RLSP is read from rlsp_dev with exact
 *             FP32 trilinear weights (border 0); with the records, runs
 *             through flat cells are added at once.
 * raw_work_dev and wet_dev hold n_beams x V floats; raw_work_dev receives
 * the unsmoothed WET.  status_dev (nullable) is one device int that is
 * OR-ed with PB_ERR_RAY_CAP if a ray reaches its step cap. */
PbStatus pb_wet(const float *rlsp_dev, PbTexture tex, const PbGrid *grid,
                const PbBeamGeom *beams, int n_beams, float *raw_work_dev,
                float *wet_dev, int *status_dev, void *stream);

/* pb_wet for callers that cannot allocate device memory (code inside a
 * framework that owns the device pool, such as an XLA/JAX custom call, or a
 * plug-in handed only its input and output buffers).  No counterpart in the
 * reference.  Same arguments and result as pb_wet, without raw_work_dev:
 * the unsmoothed WET goes to a fixed work array inside this library of
 * PB_NOALLOC_MAX_WET_FLOATS floats (32 MiB per GPU, held until exit);
 * n_beams x V above that is rejected with PB_ERR_INVALID.  The call
 * allocates nothing (tex, if non-zero, comes from pb_texture_create made
 * earlier; tex = 0 needs nothing else).  Its first call on a device looks
 * up the array's device address.  All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
#define PB_NOALLOC_MAX_WET_FLOATS (8u * 1024u * 1024u)
PbStatus pb_wet_noalloc(const float *rlsp_dev, PbTexture tex, const PbGrid *grid,
                        const PbBeamGeom *beams, int n_beams, float *wet_dev,
                        int *status_dev, void *stream);

/* The lateral-smoothing sample table that pb_wet builds for beam `beam` of
 * the n_beams given, on the host (no GPU needed).  No counterpart in the
 * reference: it exposes how the smoothing (IMPTClasses.cu:166-198) picks
 * its samples, for tests and inspection.  For direction d (angle d*pi/3)
 * and radius r+1 mm, sample (d, r) of voxel (i, j, k) is, along axis a,
 * at index i_a + floor(hh[(d*9 + r)*3 + a]), or one more where bit 3r+a of
 * tmask[d] is set (a half-voxel tie, decided per voxel in the reference's
 * FP32 order); off[d*9 + r] is the linear offset of the unflagged position.
 * Voxels with margin[a] <= i_a <= n_a - 1 - margin[a] have every candidate
 * inside the grid.  Sizes: off 54, hh 162, tmask 6, margin 3. */
PbStatus pb_smooth_table(const PbGrid *grid, const PbBeamGeom *beams, int n_beams, int beam,
                         int *off, float *hh, unsigned *tmask, int *margin);

/* The cosines and sines of the six smoothing directions (angle d*pi/3) as
 * the smoothing kernels use them: the reference forms them on the device
 * with CUDA's sincosf of the FP32 angle (IMPTClasses.cu:175-177), and where
 * a sample lies on a half-voxel their last bit decides which voxel it
 * reads.  Runs a one-thread kernel on the current device and copies the
 * twelve values back (synchronous).  No counterpart in the reference: for
 * tests and inspection. */
PbStatus pb_smooth_dirs(float cos_out[6], float sin_out[6]);

/* Forward pencil-beam dose of a plan (IMPTClasses.cu:204-271) for all of
 * its beams in one launch.  wet_dev: n_beams x V (cm).  layers_dev: all
 * layers, beam-major.  spot_geo_dev: PB_SPOT_GEO_FLOATS per spot, mu_dev:
 * one weight per spot, both in sorted (layer) order.  dose_dev (V) receives
 * scale * sum over beams; beam_dose_dev (nullable, n_beams x V) receives
 * scale * each beam's dose.  Per-voxel sums are compensated. */
PbStatus pb_dose(const PbGrid *grid, const PbBeam *beams, int n_beams,
                 const float *wet_dev, const PbLayer *layers_dev,
                 const float *spot_geo_dev, const float *mu_dev, float scale,
                 float *dose_dev, float *beam_dose_dev, void *stream);

/* Culling bounds of every layer of every beam (the fields after `energy`
 * of PbLayer), computed on the device from the spot geometry and the beam
 * models; call it once after the layers and spot geometry are on the
 * device (and again if either changes).  With bound_ok set, pb_dose,
 * pb_dose_adjoint and the batch kernels skip a layer for a voxel tile when
 * no spot of the layer can pass their per-spot cull there; the results
 * are the same as without the bounds.  No counterpart in the reference. */
PbStatus pb_layer_bounds(const PbBeam *beams, int n_beams, PbLayer *layers_dev,
                         const float *spot_geo_dev, void *stream);

/* pb_dose_adjoint and, beside it, the derivatives with respect to each
 * spot's position (x, y at the isocentre plane, mm): grad_x_dev[s] =
 * scale * sum_v dobj_dose_dev[v] * d dose[v] / d x_s, the same for y, in
 * sorted spot order; grad_dev (nullable) receives the spot-weight gradient.
 * Needs the spot weights (mu_dev).  No counterpart in the reference. */
PbStatus pb_dose_adjoint_positions(const PbGrid *grid, const PbBeam *beams, int n_beams,
                                   const float *wet_dev, const PbLayer *layers_dev,
                                   const float *spot_geo_dev, const float *mu_dev,
                                   const float *dobj_dose_dev, float scale, float *grad_dev,
                                   float *grad_x_dev, float *grad_y_dev, void *stream);

/* ------------------------------------------------------- measurement */

/* What the forward pencil-beam sum issues, counted with its own culling
 * decisions (no dose is computed): count_dev[0] = SFU exp2 operations,
 * count_dev[1] = spot-voxel evaluations (each surviving spot against the
 * 512 voxel slots of a tile).  With a time, count_dev[0] gives the SFU
 * roofline fraction of pb_dose.  No counterpart in the reference. */
PbStatus pb_count_evaluated(const PbGrid *grid, const PbBeam *beams, int n_beams,
                            const float *wet_dev, const PbLayer *layers_dev,
                            const float *spot_geo_dev, unsigned long long *count_dev,
                            void *stream);

/* As pb_count_evaluated, for what pb_dose_adjoint issues on the field
 * dobj_dose_dev with this scale: the tiles whose scale * dObj/dD is zero at
 * every voxel are skipped, as the adjoint skips them, and the count follows
 * the adjoint's kernel family.  No counterpart in the reference. */
PbStatus pb_count_evaluated_adjoint(const PbGrid *grid, const PbBeam *beams, int n_beams,
                                    const float *wet_dev, const PbLayer *layers_dev,
                                    const float *spot_geo_dev, const float *dobj_dose_dev,
                                    float scale, unsigned long long *count_dev, void *stream);

/* Measured SFU exp2 throughput of the current device (operations/s): a
 * fixed kernel of independent exp2 chains on every SM, best of three
 * timed runs.  Synchronises with the stream.  No counterpart in the
 * reference. */
PbStatus pb_measure_ex2_rate(double *ops_per_s, void *stream);

/* Page-lock an existing host range in place (cudaHostRegister), so that
 * copies from it are asynchronous DMA, and release it again.  A failure
 * leaves no pending CUDA error behind.  The range must stay allocated until
 * it is unregistered, and no copy from it may be in flight then.  No
 * counterpart in the reference (it copies from pageable memory on every
 * call). */
PbStatus pb_host_register(void *host_ptr, size_t bytes);
PbStatus pb_host_unregister(void *host_ptr);

/* Forward kernel shapes the autotuner chooses from, in two families:
 * "t<threads>_v<voxels per thread>_c<k>" works on 8x8x8 voxel tiles, each
 * thread evaluating its voxels one by one; "l8x<TY>x<TZ>_c<k>" works on
 * 8 x TY x TZ tiles, each thread a line of 8 voxels along x whose squared
 * distances to a spot's axis are one quadratic; k is the spots each thread
 * culls per compaction round.  pb_dose, pb_dose_adjoint and
 * pb_count_evaluated use pb_dose_variant_default().  No counterpart in the
 * reference (its kernel has one shape, CudaClasses.cuh:14). */
int pb_dose_variant_count(void);
int pb_dose_variant_default(void);
const char *pb_dose_variant_name(int variant);
PbStatus pb_dose_variant(const PbGrid *grid, const PbBeam *beams, int n_beams,
                         const float *wet_dev, const PbLayer *layers_dev,
                         const float *spot_geo_dev, const float *mu_dev, float scale,
                         float *dose_dev, int variant, void *stream);

/* ------------------------------------------------------------ batch */

/* One plan of a batch, as its caller holds it on the device.  beams[]
 * index into the plan's own layers_dev / spot_geo_dev / mu_dev; wet_dev and
 * raw_work_dev hold n_beams x V floats; tex (or rlsp_dev when tex == 0)
 * is the plan's RLSP. */
typedef struct {
    PbGrid grid;
    int n_beams;
    PbBeam beams[PB_MAX_BEAMS];
    const float *rlsp_dev;
    PbTexture tex;
    float *raw_work_dev;
    float *wet_dev;
    const PbLayer *layers_dev;
    const float *spot_geo_dev;
    const float *mu_dev;
    float scale;
    float *dose_dev;
} PbBatchPlan;

/* Sizes of a prepared batch, filled by pb_batch_setup. */
typedef struct {
    long long n_bricks;     /* WET work: 8x4x4-voxel bricks over all (plan, beam) */
    long long n_tiles;      /* dose work: 8x8x8 tiles over all plans              */
    int n_wet_items;        /* (plan, beam) records                              */
    int n_plans;
} PbBatchInfo;

#define PB_BATCH_WET  1     /* recompute every plan's WET                       */
#define PB_BATCH_DOSE 2     /* recompute every plan's dose                      */

/* Device work space for a batch of n_plans: plan records and the queue. */
size_t pb_batch_work_size(int n_plans);

/* Writes the batch's records into work_dev (synchronous; not for use
 * inside a stream capture).  Plans are ordered by estimated cost per tile,
 * most expensive first. */
PbStatus pb_batch_setup(const PbBatchPlan *plans, int n_plans, void *work_dev,
                        PbBatchInfo *info, void *stream);

/* Runs a prepared batch: the WET pass of every (plan, beam) in one launch
 * of 8x4x4 bricks, then one persistent forward launch of blocks_per_sm
 * blocks per SM that take (plan, tile) items from a queue in work_dev.
 * No allocation and no host synchronisation: it can be captured in a CUDA
 * graph once and replayed.  Concurrent runs on one work_dev race. */
PbStatus pb_batch_run(const PbBatchInfo *info, void *work_dev, int flags, int variant,
                      int blocks_per_sm, int *status_dev, void *stream);

/* Tile order for pb_dose_ordered and pb_dose_adjoint_ordered.  The voxel
 * tiles of the default kernel shape differ in work by more than two orders
 * of magnitude (a tile every beam crosses near the target against one no
 * spot reaches), and a launch that starts its longest tiles late ends on a
 * few of them while the other SMs idle.  pb_tile_order estimates each
 * tile's work from the WET and the layers (the layers the dose kernels keep
 * for it and their spots within reach) and writes the tile indices, most
 * expensive first, into order_dev (pb_tile_order_count ints).  work_dev:
 * pb_tile_order_work_size bytes of scratch.  Stream-ordered, no
 * allocation.  The order depends on the WET: compute it again when the WET
 * changes (a stale order gives the same results, only its speed-up is
 * lost).  Tile index o is raster order, x fastest: with the tile extent
 * (tx, ty, tz) voxels from pb_tile_order_tile and nx8 = ceil(nx / tx),
 * nty = ceil(ny / ty), tile o covers z slab o / (nx8 * nty).  An order
 * entry outside [0, count) is skipped: an order padded with -1 runs only
 * the tiles it lists and leaves the other voxels' doses unwritten.  No
 * counterpart in the reference. */
long long pb_tile_order_count(const PbGrid *grid);
PbStatus pb_tile_order_tile(int *tile_voxels);   /* 3 ints: x, y, z extent */
size_t pb_tile_order_work_size(const PbGrid *grid);
PbStatus pb_tile_order(const PbGrid *grid, const PbBeam *beams, int n_beams,
                       const float *wet_dev, const PbLayer *layers_dev, void *work_dev,
                       int *order_dev, void *stream);
/* pb_dose and pb_dose_adjoint with the default shape's tiles taken in the
 * order of order_dev (from pb_tile_order for this grid; NULL: the default
 * order).  Each voxel's dose is the same bits as pb_dose's. */
PbStatus pb_dose_ordered(const PbGrid *grid, const PbBeam *beams, int n_beams,
                         const float *wet_dev, const PbLayer *layers_dev,
                         const float *spot_geo_dev, const float *mu_dev, float scale,
                         float *dose_dev, float *beam_dose_dev, const int *order_dev,
                         void *stream);
PbStatus pb_dose_adjoint_ordered(const PbGrid *grid, const PbBeam *beams, int n_beams,
                                 const float *wet_dev, const PbLayer *layers_dev,
                                 const float *spot_geo_dev, const float *dobj_dose_dev,
                                 float scale, float *grad_dev, const int *order_dev,
                                 void *stream);

/* Adjoint of pb_dose: grad_dev[s] = scale * sum_v dobj_dose_dev[v] * K(v,s)
 * for every spot s, where K(v,s) is the dose per unit weight of spot s at
 * voxel v.  Matrix-free: footprints are recomputed.  grad_dev is
 * overwritten. */
PbStatus pb_dose_adjoint(const PbGrid *grid, const PbBeam *beams, int n_beams,
                         const float *wet_dev, const PbLayer *layers_dev,
                         const float *spot_geo_dev, const float *dobj_dose_dev,
                         float scale, float *grad_dev, void *stream);
/* pb_dose_adjoint with the kernel family of forward shape `variant`
 * (pb_dose_variant_name): the same gradient, to float rounding. */
PbStatus pb_dose_adjoint_variant(const PbGrid *grid, const PbBeam *beams, int n_beams,
                                 const float *wet_dev, const PbLayer *layers_dev,
                                 const float *spot_geo_dev, const float *dobj_dose_dev,
                                 float scale, float *grad_dev, int variant, void *stream);

/* Quadratic objective sum_v w_v (D_v - P_v)^2, reduced in FP64 into
 * *obj_dev, and its gradient 2 w_v (D_v - P_v) into resid_dev (nullable).
 * work_dev holds pb_objective_work_size() bytes. */
size_t pb_objective_work_size(void);
PbStatus pb_objective(const float *dose_dev, const float *presc_dev,
                      const float *weight_dev, int64_t n, double *obj_dev,
                      float *resid_dev, void *work_dev, void *stream);

/* Dense spot-voxel pair count of a plan: sum over beams and layers of
 * |{v : 10*WET(v) <= 1.1*R80}| * spots (the reference kernel's work,
 * IMPTClasses.cu:222-226,255).  count_dev is one uint64, overwritten. */
PbStatus pb_count_pairs(const PbGrid *grid, const PbBeam *beams, int n_beams,
                        const float *wet_dev, const PbLayer *layers_dev,
                        unsigned long long *count_dev, void *stream);

/* ---------------------------------------------------- host drop-in level */

/* proton_raytrace_cuda: smoothed WET of one beam from host RLSP
 * (IMPTClasses.cu:274-299 via dosemodule.cu:104-201), sampled through a
 * texture as the reference does.  dims are the numpy shape (nz, ny, nx). */
PbStatus pb_proton_raytrace_host(int gpu_id, double vsadx, double vsady,
                                 const float *rlsp, const int64_t dims[3],
                                 float spacing, const float origin[3],
                                 const float iso[3], double gantry_deg,
                                 double couch_deg, float *wet_out);

/* proton_spot_cuda: dose of one beam from host WET and spots
 * (IMPTClasses.cu:301-340 via dosemodule.cu:243-374). */
PbStatus pb_proton_spot_host(int gpu_id, double vsadx, double vsady,
                             const float *dvp, const float *depths,
                             const float *sigmas, const float *idds,
                             int n_energies, int lut_len, int dvp_len,
                             const float *wet, const int64_t dims[3],
                             float spacing, const float origin[3],
                             const float iso[3], double gantry_deg,
                             double couch_deg, const float *spot_list,
                             int n_spots, float *dose_out);

#ifdef __cplusplus
}
#endif

#endif /* PB_B200_H */
