// pb_internal.h -- declarations shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/pb_b200.h"
#include "pb_device.cuh"

namespace pb {

// Records an error message for pb_last_error() and returns `code`.
PbStatus set_error(PbStatus code, const char *fmt, ...);

// Checks the last launch; on failure records the CUDA error text.
PbStatus check_launch(const char *what);
PbStatus check_cuda(cudaError_t e, const char *what);

// cos/sin of the six smoothing directions, angle i*pi/3 in FP32 as the
// reference forms it (IMPTClasses.cu:177), evaluated on the host.
void smooth_dirs(float *c, float *s);

int ray_step_cap(const PbGrid &g);

// The smoothing directions as the smoothing kernels form them on the
// current device (CUDA's sincosf), copied to the host.
PbStatus device_smooth_dirs(float *c, float *s);

PbStatus launch_rlsp(const float *hu, int64_t n, const double *xh,
                     const double *yh, int m, float *out, cudaStream_t st);

// The argument checks of the WET entry points (pb_wet, pb_wet_noalloc):
// grid, input (RLSP pointer or texture), beams and output.
PbStatus check_wet_args(const float *rlsp_dev, uint64_t tex, const PbGrid *grid,
                        const PbBeamGeom *beams, int n_beams, const float *wet_dev);

PbStatus launch_wet(const float *rlsp, cudaTextureObject_t tex, const float2 *rec,
                    const PbGrid &g, const PbBeamGeom *beams, int n_beams, float *raw,
                    float *wet, int *status, cudaStream_t st);

// Batched WET pass (pb_wet.cu): one record per (plan, beam).
// The smoothing sample table of one beam (pb_wet.cu), as the WET launch
// builds it: off[6][9], hh[6][9][3], tmask[6], margin[3].
void smooth_table_host(const PbGrid &g, const PbBeamGeom *beams, int n_beams, int beam,
                       int *off, float *hh, unsigned *tmask, int *margin);

size_t batch_wet_size();
long long fill_batch_wet(void *items_host, int first, const PbGrid &g, const PbBeamGeom *beams,
                         int n_beams, const float *rlsp, cudaTextureObject_t tex,
                         const float2 *rec, float *raw, float *wet, long long brick_start);
PbStatus launch_wet_batch(const void *items_dev, int n_items, long long n_bricks, int *status,
                          cudaStream_t st);

PbStatus texture_create(const float *rlsp, const PbGrid &g, uint64_t *out, cudaStream_t st,
                        bool with_texture = true);
bool texture_samples(uint64_t h);   // a texture (not a records-only handle)
PbStatus texture_update(uint64_t h, const float *rlsp, cudaStream_t st);
bool texture_matches(uint64_t h, const PbGrid &g);
cudaTextureObject_t texture_object(uint64_t h);
const float2 *texture_cells(uint64_t h);
void texture_destroy(uint64_t h);

PbStatus launch_dose(const PbGrid &g, const PbBeam *beams, int n_beams,
                     const float *wet, const PbLayer *layers,
                     const float *geo, const float *mu, float scale,
                     float *dose, float *beam_dose, cudaStream_t st, int variant = -1,
                     const int *order = nullptr);

// variant < 0 selects the default forward shape (dose_variant_default);
// the adjoint and the operation count use the kernel family of `variant`.
int dose_variant_default();
int dose_variant_count();
const char *dose_variant_name(int v);
int dose_variant_threads(int variant);

// Batched forward (pb_dose.cu): device records of the plans of a batch.
struct BatchDose;
size_t batch_dose_size();
long long plan_tiles(const PbGrid &g);
void fill_batch_dose(BatchDose &D, const PbGrid &g, const PbBeam *beams, int n_beams,
                     float scale, const float *wet, const PbLayer *layers, const float *geo,
                     const float *mu, float *dose, long long tile_start);
PbStatus launch_dose_batch(const void *plans_dev, int n_plans, long long n_items,
                           unsigned long long *counter, int variant, int blocks,
                           cudaStream_t st);

PbStatus launch_adjoint(const PbGrid &g, const PbBeam *beams, int n_beams,
                        const float *wet, const PbLayer *layers,
                        const float *geo, const float *w, float scale,
                        float *grad, cudaStream_t st, int variant = -1,
                        const int *order = nullptr);
long long tile_order_count(const PbGrid &g);
void tile_order_tile(int *voxels);
size_t tile_order_work_size(const PbGrid &g);
PbStatus launch_tile_order(const PbGrid &g, const PbBeam *beams, int n_beams, const float *wet,
                           const PbLayer *layers, void *work, int *order, cudaStream_t st);

PbStatus launch_objective(const float *dose, const float *presc,
                          const float *weight, int64_t n, double *obj,
                          float *resid, void *work, cudaStream_t st);
size_t objective_work_size();

PbStatus launch_adjoint_positions(const PbGrid &g, const PbBeam *beams, int n_beams,
                                  const float *wet, const PbLayer *layers, const float *geo,
                                  const float *mu, const float *w, float scale, float *grad,
                                  float *grad_x, float *grad_y, cudaStream_t st);
PbStatus launch_layer_bounds(const PbBeam *beams, int n_beams, PbLayer *layers,
                            const float *geo, cudaStream_t st);
PbStatus launch_count_evaluated(const PbGrid &g, const PbBeam *beams, int n_beams,
                                const float *wet, const PbLayer *layers, const float *geo,
                                unsigned long long *count, cudaStream_t st, int variant = -1,
                                const float *wfield = nullptr, float scale = 1.0f);
PbStatus measure_ex2_rate(double *ops_per_s, cudaStream_t st);
PbStatus launch_count_pairs(const PbGrid &g, const PbBeam *beams, int n_beams,
                            const float *wet, const PbLayer *layers,
                            unsigned long long *count, cudaStream_t st);

}  // namespace pb
