/*
 * yg.h — C-ABI of the B200 visibility gridder.
 *
 * A drop-in GPU back end for yandasoft's IVisGridder path
 * (askap/gridding/IVisGridder.h:64-140) for the SphFunc, WProject, WStack and
 * AWProject gridders, plus a W-stacking + W-projection hybrid.  A C++
 * IVisGridder subclass on the yandasoft side unpacks its accessor into a
 * yg_chunk and forwards each virtual call to the function named beside it
 * below.
 *
 * Conventions
 *   - Every function returns 0 (YG_OK) or a YG_ERR_* code; yg_last_error()
 *     returns the message of the last failure on the calling thread.  The shim
 *     rethrows it as askap::AskapError, as ASKAPCHECK would.
 *   - Cubes are the reference's casacore layout: (nrow, nchan, npol),
 *     column-major (row fastest).  Complex values are interleaved float pairs.
 *   - Images are (nx, ny, npol, nchan) column-major float, the unpadded shape.
 *   - A handle is not thread-safe; use one handle per host thread (clone).
 *     Each handle owns one CUDA stream and its device memory.
 *   - Host buffers stay caller-owned.  With on_device = 1 every pointer of a
 *     chunk (except pointing) is a device pointer on the current device.
 */
#ifndef YG_H
#define YG_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  YG_OK = 0,
  YG_ERR_ARG = 1,
  YG_ERR_CUDA = 2,
  YG_ERR_FRAC = 3,
  YG_ERR_WRANGE = 4,
  YG_ERR_WEIGHT = 5,
  YG_ERR_CINDEX = 6,
  YG_ERR_SUPPORT = 7,
  YG_ERR_STATE = 8,
  YG_ERR_UNSUPPORTED = 9,
  YG_ERR_FREQ = 10,
  YG_ERR_TIMEOUT = 11,
  YG_ERR_NOMEM = 12
};

typedef struct yg_gridder yg_gridder;
typedef struct yg_plan yg_plan;

/* scimath::Axes as the gridder reads it (TableVisGridder::initialiseCellSize,
 * getImageCentre, getTangentPoint, FrequencyMapper::setupImage). */
typedef struct yg_axes {
  double cell[2];        /* direction-axis increments, radians */
  double centre[2];      /* image centre (ra, dec), radians */
  double tangent[2];     /* tangent point (ra, dec), radians */
  int32_t has_freq;      /* 1 if the image has a FREQUENCY axis */
  int32_t reserved;
  double freq_start;     /* Hz of the first image channel */
  double freq_end;       /* Hz of the last image channel */
} yg_axes;

/* One accessor chunk (accessors::IConstDataAccessor / IDataAccessor). */
typedef struct yg_chunk {
  int64_t nrow;
  int32_t nchan;
  int32_t npol;
  const double* uvw;       /* nrow x 3 rotatedUVW(tangent), metres, row-major */
  const double* delay;     /* nrow uvwRotationDelay(tangent, centre) or NULL */
  const double* freq;      /* nchan, Hz */
  float* vis;              /* complex cube; grid reads it, degrid adds into it */
  const float* noise;      /* complex cube or NULL (noise 1) */
  const uint8_t* flag;     /* cube or NULL */
  const int32_t* feed1;    /* nrow or NULL (AWProject, PSF feed selection) */
  const double* pointing;  /* HOST nrow x 2 pointingDir1 (ra, dec) or NULL */
  int32_t on_device;       /* 1: uvw, delay, freq, vis, noise, flag, feed1 are device pointers */
  int32_t reserved;
} yg_chunk;

/* Last error message of the calling thread. */
const char* yg_last_error(void);

/* VisGridderFactory::make (askap/gridding/VisGridderFactory.cc:112-285).
 * parset: "key = value" lines, keys as in a cimager parset with or without the
 * "Cimager." prefix ("gridder = WProject", "gridder.WProject.wmax = 5000" ...). */
int yg_create(const char* parset, yg_gridder** out);

/* IVisGridder::clone (IVisGridder.h:77). */
int yg_clone(const yg_gridder* g, yg_gridder** out);

void yg_destroy(yg_gridder* g);

/* IVisGridder::initialiseGrid (TableVisGridder.cc:997-1030).  dopsf: grid the
 * weights (PSF); dopcf: the preconditioner function (weights without the MFS
 * factor, conjugate CF on one half of the uv plane, no sums of weights,
 * TableVisGridder.cc:825-851); not both at once. */
int yg_initialise_grid(yg_gridder* g, const yg_axes* axes, int32_t nx, int32_t ny, int32_t npol, int32_t nchan,
                       int32_t dopsf, int32_t dopcf);

/* IVisGridder::grid (TableVisGridder.cc:908-913 -> generic(acc, false)). */
int yg_grid(yg_gridder* g, const yg_chunk* chunk);

/* IVisGridder::finaliseGrid (TableVisGridder.cc:1109-1236; WStackVisGridder.cc:216-295). */
int yg_finalise_grid(yg_gridder* g, float* image, int32_t on_device);

/* IVisGridder::finaliseWeights (TableVisGridder.cc:1255-1284). */
int yg_finalise_weights(yg_gridder* g, float* weights, int32_t on_device);

/* IVisGridder::initialiseDegrid (TableVisGridder.cc:1286-1319; WStackVisGridder.cc:297-337). */
int yg_initialise_degrid(yg_gridder* g, const yg_axes* axes, int32_t nx, int32_t ny, int32_t npol, int32_t nchan,
                         const float* image, int32_t on_device);

/* IVisGridder::degrid (TableVisGridder.cc:898-902 -> generic(acc, true)); adds
 * the model visibilities into chunk->vis. */
int yg_degrid(yg_gridder* g, yg_chunk* chunk);

/* IVisGridder::finaliseDegrid (TableVisGridder.cc:1364-1372). */
int yg_finalise_degrid(yg_gridder* g);

/* IVisGridder::customiseForContext (TableVisGridder.cc:1381-1405). */
int yg_customise_for_context(yg_gridder* g, const char* context);

/* IVisGridder::initVisWeights with VisWeightsMultiFrequency(reffreq)
 * (VisGridderFactory.cc:265-272). */
int yg_init_vis_weights_mfs(yg_gridder* g, double reffreq);

/* IVisGridder::isModelEmpty (TableVisGridder.cc:1466-1469). */
int yg_is_model_empty(const yg_gridder* g, int32_t* empty);

/* ---- inspection (itsSupport, itsOverSample, itsConvFunc, itsSumWeights) ---- */
int yg_get_support(const yg_gridder* g, int32_t* support, int32_t* oversample, int32_t* ncf);
/* CF cache: sizes[ncf] (2S+1), offsets[ncf] (complex elements), data (complex). */
int yg_get_cf(const yg_gridder* g, int32_t* sizes, int64_t* offsets, float* data, int64_t data_capacity);
/* itsConvFuncOffsets: 2 ints per plane; *n receives the number of planes. */
int yg_get_cf_offsets(const yg_gridder* g, int32_t* offsets, int32_t capacity, int32_t* n);
/* itsSumWeights (rows, npol, nchan) column-major; *nrows receives rows. */
int yg_get_sum_weights(const yg_gridder* g, double* out, int64_t capacity, int32_t* nrows);
/* itsGrid: ngrids x (nx, ny, npol, nchan) complex, padded shape. */
int yg_get_grid(const yg_gridder* g, float* out, int64_t capacity_complex, int32_t* ngrids);
/* padded grid shape */
int yg_get_shape(const yg_gridder* g, int32_t* nx, int32_t* ny, int32_t* npol, int32_t* nchan);
/* stats: samples/taps gridded, samples/taps degridded, ms grid, ms degrid, ms CF, CF planes built */
int yg_get_stats(const yg_gridder* g, double* out8);
/* device time of the tap kernels: k_grid ms, k_grid calls, k_degrid ms, k_degrid calls */
int yg_get_kernel_times(const yg_gridder* g, double* out4);
/* number of this library's own kernel launches so far (process-wide) */
int64_t yg_kernel_launch_count(void);
/* builds the convolution functions for the current axes without data
 * (SphFunc, WProject, WStack; AWProject builds from data). */
int yg_build_cf(yg_gridder* g);

/* ---- plans: bin a chunk once, grid/degrid it many times (major cycle) ---- */
int yg_plan_create(yg_gridder* g, const yg_chunk* chunk, yg_plan** out);
int yg_plan_grid(yg_gridder* g, const yg_plan* plan, const yg_chunk* chunk);
int yg_plan_degrid(yg_gridder* g, yg_plan* plan, yg_chunk* chunk);
/* on-grid samples and work items of a plan */
int yg_plan_info(const yg_plan* plan, int64_t* nvalid, int32_t* nitems, int32_t* tile);
/* per sample (row + nrow*chan order): grid position iu, iv (with the CF
 * offset applied; 0 off-grid), CF index, status (0 unused, 1 w out of range,
 * 2 off the grid, 3 gridded) */
int yg_plan_samples(const yg_gridder* g, const yg_plan* plan, int32_t* iu, int32_t* iv, int32_t* cfi,
                    uint8_t* status);
void yg_plan_destroy(yg_plan* plan);

/* ---- tuning ---- */
int yg_set_tile(yg_gridder* g, int32_t tile);      /* 0 = automatic */
int yg_set_item_size(yg_gridder* g, int32_t vmax); /* samples per work item */
/* k_grid thread layout: 0 or 1 the default, 2 and 3 halve / quarter the tap
 * threads (each steps down twice / four times the rows); YG_ERR_UNSUPPORTED
 * at the next grid call when the CF width has no such layout.  Adding 16
 * keeps each thread's running tap sums in registers while consecutive
 * samples cover the same cell (layouts of at most 8 rows per thread); adding
 * 32 as well orders each tile's samples by position before CF for gridding
 * (plans made afterwards keep both orders) and reads the taps through L2;
 * adding 64 orders them by CF plane, then position, then oversampling offset
 * and stages each plane's offsets in shared memory once (16-wide CFs), and
 * 128 with it keeps that kernel's tile in global memory (two CTAs per SM).
 * Adding 256 degrids 16-wide CFs with the CF read per tap from the segment
 * ring (k_degrid_t) instead of the default register-held CF column; adding
 * 512 has the default degrid one sample per half-warp pass instead of two. */
int yg_set_grid_variant(yg_gridder* g, int32_t variant);
int yg_synchronize(yg_gridder* g);
/* the cudaStream_t every kernel of this handle is launched on */
int yg_get_stream(yg_gridder* g, void** stream);

/* ---- degridding without device allocation ----
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * an application that fixes each GPU's memory budget when it starts and
 * forbids any later allocation (so that a long-running imaging service cannot
 * fail half way through a major cycle for lack of memory), or a host
 * framework whose own pool allocator owns the device's memory.
 * Same semantics as yg_degrid for a device-resident chunk (on_device = 1):
 * the model visibilities are added into chunk->vis.  The gridder must have
 * its convolution functions built (yg_build_cf, or one earlier yg_degrid) and
 * its model grid initialised (yg_initialise_degrid); both stay owned by the
 * handle.  SphFunc, WStack, WProject and WStackWProject with the tabulated
 * CFs; AWProject (CFs built per chunk) and the learned CF forms return
 * YG_ERR_UNSUPPORTED.  Every temporary of the call lives in one static device
 * array of about 60 MB that each GPU loading the library holds until exit;
 * the call takes at most 2^20 rows x channels (YG_ERR_ARG beyond that), 1, 2
 * or 4 polarisations and 65536 channels, and allocates nothing.  The array's
 * device address is looked up the first time the call runs on a device.  All
 * calls share the array: calls that overlap on the GPU (other streams, other
 * host threads) race on it and must be serialised by the caller.  Like
 * yg_degrid, the call reads the chunk's frequencies back to the host and
 * waits for the handle's stream before it returns. */
int yg_degrid_noalloc(yg_gridder* g, yg_chunk* chunk);

/* ---- learned convolution function ----
 * No counterpart in the reference.  A sinusoidal MLP (5 inputs: the tap's
 * continuous uv offset, w, frequency, beam; 4 hidden layers of 64; real and
 * imaginary part out; FP16 weights, FP32 accumulation) trained on the GPU on
 * the gridder's own tabulated CFs (WProjectVisGridder::initConvolutionFunction,
 * WProjectVisGridder.cc:435-726, or AWProjectVisGridder::initConvolutionFunction,
 * AWProjectVisGridder.cc:259-611) and evaluated inside the grid and degrid
 * kernels in place of the table.  WProject, WStackWProject and AWProject; an
 * AWProject handle trains after its CFs are built (every beam of maxfeeds seen,
 * one field), with each plane's channel frequency and beam as the f and b
 * inputs, and nwplanes_train is ignored for it. */
typedef struct {
  int64_t ntrain;          /* training taps drawn from the tabulated CFs */
  int32_t batch;           /* taps per Adam step */
  int32_t steps;           /* Adam steps */
  double lr;               /* peak learning rate (cosine decay to lr / 20) */
  uint64_t seed;
  int32_t nwplanes_train;  /* > the gridder's nwplanes: train on a denser table of this many
                              planes over the same w range (built and released by the call) */
  int32_t reserved;
} yg_learn_params;

typedef struct {
  double final_loss;       /* mean squared tap error of the last minibatch, in units of the largest tap */
  float train_ms;          /* GPU time of the Adam steps */
  int32_t steps;
  float scale;             /* the largest |tap| (network output unit) */
  double cf_table_bytes;   /* device bytes of the tabulated CFs (packed + padded copies) */
  double network_bytes;    /* bytes of the FP16 network */
} yg_learn_report;

int32_t yg_mlp_nparams(void);
int yg_learned_train(yg_gridder* g, const yg_learn_params* p, yg_learn_report* rep);
/* 0: tabulated CFs (default); 1: the learned network at the tabulated offsets
 * and w planes; 2: the learned network at every sample's own fractional
 * offsets and w (continuous, no oversampling or w-plane quantisation; not for
 * AWProject: YG_ERR_UNSUPPORTED).  YG_ERR_STATE before training. */
int yg_set_cf_form(yg_gridder* g, int32_t form);
int yg_learned_get_params(yg_gridder* g, float* params, float* scale);
int yg_learned_set_params(yg_gridder* g, const float* params, float scale);
/* the network's loss scale * sum |y - t|^2 over n taps and its gradient with
 * respect to params (FP32 master weights; the forward pass uses them rounded
 * to FP16), on host arrays: x is n x 5, t is n x 2, grad has yg_mlp_nparams() */
int yg_mlp_loss_grad(const float* params, const float* x, const float* t, int64_t n, float scale, float* grad,
                     double* loss);
/* y (n x 2) of the network with params rounded to FP16, host arrays */
int yg_mlp_eval(const float* params, const float* x, int64_t n, float* y);

/* The plan builder's device primitives on host arrays (no reference
 * counterpart: the reference grids samples in accessor order and sorts
 * nothing).  yg_sort_pairs sorts (keys[i], vals[i]) in place by bits
 * [0, end_bit) of the key, stably; yg_scan_i32 writes the inclusive (or, with
 * exclusive != 0, exclusive) scan of in under op 0 = sum, 1 = min, 2 = max;
 * in == out is allowed.  n < 2^31. */
int yg_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n, int32_t end_bit);
int yg_scan_i32(const int32_t* in, int32_t* out, int64_t n, int32_t op, int32_t exclusive);

/* ---- major cycle as a CUDA graph ----
 * The caller's major-cycle sequence of ImageFFTEquation::calcImagingEquations
 * (ImageFFTEquation.cc:437-479) for n independent imaging instances: instance
 * i degrids the model held by degridders[i] (after yg_initialise_degrid) into
 * model visibilities, subtracts them from the observed visibilities of
 * chunks[i] (device-resident, on_device = 1) and grids the residual with
 * gridders[i] (after yg_initialise_grid).  yg_cycle_create bins every chunk,
 * runs one cycle uncaptured (sizing every buffer) and records the n
 * sequences, each on a branch of its own, into one CUDA graph; yg_cycle_run
 * replays it `cycles` times.  Between runs the caller may load a new model
 * (yg_initialise_degrid with an image of the same shape) and re-initialise
 * the residual grids (yg_initialise_grid): buffers keep their addresses.
 * The handles, chunks and arrays must outlive the cycle. */
typedef struct yg_cycle yg_cycle;
int yg_cycle_create(int32_t n, yg_gridder* const* degridders, yg_gridder* const* gridders, const yg_chunk* chunks,
                    yg_cycle** out);
/* The same with the other roles of ImageFFTEquation::calcImagingEquations
 * (ImageFFTEquation.cc:362-387, 437-479): after the residual, instance i's
 * PSF gridder (yg_initialise_grid with dopsf = 1) and preconditioner-function
 * gridder (dopcf = 1), where given, grid the same visibility buffer within
 * the same graph branch.  model and residual are required; psf and pcf may
 * be NULL. */
typedef struct yg_cycle_roles {
  yg_gridder* model;      /* degrids the model (after yg_initialise_degrid) */
  yg_gridder* residual;   /* grids the residual (after yg_initialise_grid) */
  yg_gridder* psf;        /* PSF gridder or NULL */
  yg_gridder* pcf;        /* preconditioner-function gridder or NULL */
} yg_cycle_roles;
int yg_cycle_create_roles(int32_t n, const yg_cycle_roles* roles, const yg_chunk* chunks, yg_cycle** out);
/* replays the graph `cycles` times; *gpu_ms (may be NULL) receives the GPU time */
int yg_cycle_run(yg_cycle* c, int32_t cycles, float* gpu_ms);
/* nodes of the recorded graph */
int yg_cycle_info(const yg_cycle* c, int64_t* nodes);
void yg_cycle_destroy(yg_cycle* c);

/* ---- autotuner ----
 * No counterpart in the reference.  Times a degrid + grid pass over a
 * device-resident chunk for up to max_trials candidates of (uv tile side,
 * samples per work item, k_grid thread layout) and keeps the fastest for this
 * handle and, process-wide, for every later handle whose CFs have the same
 * padded width and polarisation count.  The handle must be initialised
 * (yg_initialise_grid or yg_initialise_degrid); its grids hold extra passes
 * afterwards, so re-initialise before real use. */
typedef struct {
  int32_t tile, items, variant;   /* the choice kept */
  int32_t trials;                 /* candidates timed */
  float best_ms, default_ms;      /* degrid + grid pass with the choice / with the defaults */
  int32_t cf_width, npol;         /* the class it is kept for (padded CF width) */
} yg_tune_report;
int yg_autotune(yg_gridder* g, const yg_chunk* chunk, int32_t max_trials, yg_tune_report* rep);
/* forgets every process-wide choice */
void yg_autotune_reset(void);

#ifdef __cplusplus
}
#endif

#endif /* YG_H */
