/*
 * dba.h -- C ABI of the B200 dynamic-block-activation (DBA) stencil engine.
 *
 * The reference (zhangruoyao68/DBA) has no library API: each model is a
 * program that reads ./Input.txt, allocates unified-memory arrays, runs a
 * fixed kernel sequence per time step and writes .vtk/.out files.  These
 * entry points replace the pieces of those programs, so a host program (the
 * dba_run executable in this repository, the Python package, or a third
 * party) can drive the same path.  Plain C types only; every function returns
 * a status code (DBA_OK or a DBA_ERR_*), never exits the process.
 *
 * Threading: one dba_ctx is used by one host thread at a time.  Each context
 * owns a CUDA stream and all of its device memory; separate contexts may run
 * concurrently.
 */
#ifndef DBA_H
#define DBA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DBA_ABI_VERSION 1

/* ---- status codes ---- */
#define DBA_OK 0
#define DBA_ERR_CONFIG 1      /* invalid or unsupported configuration */
#define DBA_ERR_CUDA 2        /* a CUDA runtime call failed */
#define DBA_ERR_NOMEM 3       /* device or host allocation failed */
#define DBA_ERR_IO 4          /* file could not be opened / parsed */
#define DBA_ERR_NONFINITE 5   /* a kernel produced NaN/inf in a state field */
#define DBA_ERR_TIMEOUT 6     /* a bounded device wait gave up */
#define DBA_ERR_STATE 7       /* call out of order (e.g. step before init) */
#define DBA_ERR_ARG 8         /* bad argument (null pointer, bad field id) */

/* ---- enumerations ---- */
#define DBA_MODEL_DENDRITE 0  /* Kobayashi p/T, example_Dendritic_growth/ */
#define DBA_MODEL_MODELB 1    /* reactive ternary Cahn-Hilliard, example_Reactive_ModelB/ */
#define DBA_MODEL_KH 2        /* 2-D compressible Euler, example_Kelvin_Helmholtz/ */

#define DBA_PREC_F64 0        /* FP64 stencils; bit-exact with the CPU restatement */
#define DBA_PREC_F32 1        /* FP32 stencils, FP64 conserved sums and tip tracking */

#define DBA_BC_PERIODIC 0     /* reference: wrap in cells and in block indices */
#define DBA_BC_ZEROFLUX 1     /* mirror (clamped) neighbours, no block wrap */

#define DBA_MODE_REGULAR 0    /* every block updated (reference mode 0) */
#define DBA_MODE_DBA 1        /* only active blocks updated (reference mode 1) */

#define DBA_IC_REFERENCE 0    /* the reference program's own initial condition */
#define DBA_IC_TANH_SEED 1    /* dendrite: tanh-profile solid seed of radius ic_radius */
#define DBA_IC_SHARP_BANDS 2  /* KH: sharp |y-0.5|<0.25 bands plus seeded white noise */
#define DBA_IC_CURAND 3       /* Model B: the reference GPU program's draw (example_Reactive_ModelB/kernel.cu:
                                 1032-1042): cuRAND's default generator (XORWOW) seeded with `seed`, three
                                 uniform-double passes for x, y, z, then Initialize (:209-211) in FP64 with
                                 separately rounded product and sum.  DBA_IC_REFERENCE for Model B is the
                                 reference CPU program's mt19937_64 stream (CPU_version/base_CPU.cpp:540-549). */

/* ---- configuration: the reference's Input.txt values plus engine options ---- */
typedef struct dba_config {
    int model;                 /* DBA_MODEL_* */
    int nx, ny, nz;            /* cells; nz == 1 selects the 2-D stencils */
    int t_total, t_freq;       /* steps and output period (used by dba_run) */
    int mode;                  /* DBA_MODE_* requested by Input.txt */
    double dt, dx, dy, dz;
    /* dendrite (example_Dendritic_growth/kernel.cu:40-64) */
    double delta, tau, epsilon, alpha, gamma, Delta, metric_p, metric_T;
    /* Model B (example_Reactive_ModelB/kernel.cu:49-87) */
    double chi_xy, chi_xz, chi_yz, chi_xb, chi_yb, chi_zb;
    int vx, vy, vz, rx, ry, rz, n, m;
    double eps_x, eps_y, eps_z, eps_phi;
    double mob_x, mob_y, mob_z, mob_phi;
    double x0, y0, z0, K, z_crit, p_gel, k_0;
    double metric_eps;         /* Model B and KH wake-up threshold (Metric_eps) */
    /* KH (example_Kelvin_Helmholtz/KH_DBA.cu:66-85) */
    double kh_gamma;           /* adiabatic index; the reference hard-codes 5/3 */
    /* engine options (not in the reference's Input.txt) */
    int block;                 /* DBA block edge in cells (4 = the reference's dendrite/Model B, 8 = KH) */
    int precision;             /* DBA_PREC_* */
    int bc;                    /* DBA_BC_* */
    int conserved;             /* Model B / KH: the Conserved/ variant (global change removed each step) */
    int ic;                    /* DBA_IC_* used by dba_init(ctx, NULL) */
    unsigned long long seed;   /* Model B noise / KH noise seed (mt19937_64) */
    double ic_radius, ic_width;/* dendrite tanh seed */
    int ic_corner;             /* dendrite tanh seed at cell (0,0,0) instead of the centre */
    double noise_amp, noise_amp_z; /* Model B: x,y and z uniform-noise amplitudes (0.05, 0.001) */
    int tiles;                 /* 1 (default): tile kernels where the shape allows -- FP32 2-D Model B on 32x32
                                  cells (nx, ny multiples of 32, block 8 or 16), KH on 16x16 cells (nx, ny
                                  multiples of 16, block 8 or 16), FP32 3-D dendrite on 32x8x8 cells (block 8,
                                  nx a multiple of 32); 2: as 1, with the FP32 2-D Model B tiles staged by
                                  bulk copies of the TMA engine (one per block segment of a staged row)
                                  instead of 16-byte cp.async pieces; 0: the one-block kernels and the
                                  four-stage KH kernels */
    double cfl;                /* KH: > 0 picks each step's dt = cfl * min(dx, dy) / max(c + |v|) on the device
                                  (tile kernel only); 0 (default): the fixed dt */
} dba_config;

typedef struct dba_ctx dba_ctx;

/* observables computed on the device at the current step */
typedef struct dba_obs {
    long step;                 /* completed steps */
    double time;               /* simulated time */
    int active_blocks[2];      /* blocks active for the NEXT step, per channel (dendrite: p, T) */
    int total_blocks;
    double tip;                /* dendrite growth_front at x = Nx/2 (NaN if no p < 0.5 found) */
    double integral[4];        /* dendrite: sum p, sum T; Model B: sum x,y,z,b; KH: sum Mass,Energy,Momx,Momy */
    double vy_mode;            /* KH: amplitude of the vy mode (Calc_Vy_mode) */
    long cell_updates;         /* active cell-updates accumulated since dba_init */
    double dt;                 /* time step the next step will take (KH with cfl > 0: set on the device) */
} dba_obs;

typedef struct dba_info {
    int nbx, nby, nbz, nb;     /* block counts */
    int dims;                  /* 2 or 3 */
    int nfields;               /* readable fields */
    int nchannels;             /* activity channels (2 for dendrite p/T, else 1) */
    size_t device_bytes;       /* device memory held by the context */
    long step;
    int grid_ctas;             /* CTAs per step launch */
    long active_block_steps;   /* blocks processed (active in any channel), summed over steps since dba_init */
    long cells_per_block;
} dba_info;

/* ---- configuration ---- */

/* Defaults of the reference's Input.txt for `model`
 * (example_Dendritic_growth/Input.txt, example_Reactive_ModelB/Input.txt,
 * example_Kelvin_Helmholtz/Input.txt) with engine options set to parity mode. */
int dba_config_default(int model, dba_config* cfg);

/* Replaces ReadInput (example_Dendritic_growth/kernel.cu:67-112,
 * example_Reactive_ModelB/kernel.cu:90-142, example_Kelvin_Helmholtz/KH_DBA.cu:88-122):
 * reads the reference's positional Input.txt grammar for `model`.  Fields not
 * in the file keep their dba_config_default values.  Lines after the
 * reference grammar may hold `key = value` engine options (block, precision,
 * bc, conserved, ic, seed, ic_radius, ic_width, ic_corner, gamma_kh,
 * noise_amp, noise_amp_z). */
int dba_parse_input(const char* path, int model, dba_config* cfg);

/* ---- lifetime ---- */

/* Replaces Allocate (example_Dendritic_growth/kernel.cu:115-135 and the
 * models' twins): validates `cfg` and allocates device state on the current
 * CUDA device. */
int dba_create(const dba_config* cfg, dba_ctx** out);

/* Replaces Initialize (example_Dendritic_growth/kernel.cu:138-178,
 * example_Reactive_ModelB/kernel.cu:173-238 with its cuRAND draw :1032-1042,
 * example_Kelvin_Helmholtz/KH_DBA.cu:1047-1130 + getConserved :335-372).
 * ic == NULL: the initial condition cfg->ic describes.  Otherwise host FP64
 * fields, each nx*ny*nz x-fastest: dendrite p,T; Model B x,y,z; KH rho,p,vx,vy.
 * All blocks start active; the step counter is reset. */
int dba_init(dba_ctx* ctx, const double* ic);
/* dba_init from FP32 host fields (no counterpart in the reference: its fields are FP64).
 * Same layout and meaning as dba_init's `ic` (non-null).  An FP32 context copies them to
 * the device as they are (page-locked host memory moves at full link speed); an FP64 context
 * or a KH context converts them to FP64 first. */
int dba_init_f32(dba_ctx* ctx, const float* ic);

/* Replaces the body of the time loop of main()
 * (example_Dendritic_growth/kernel.cu:913-990, example_Reactive_ModelB/kernel.cu:1057-1161,
 * Conserved/kernel.cu:1095-1190, example_Kelvin_Helmholtz/KH_DBA.cu:1384-1500):
 * enqueues nsteps steps in `mode` on the context's stream.  Asynchronous;
 * errors raised on the device are reported by dba_sync. */
int dba_step(dba_ctx* ctx, int nsteps, int mode);

/* Waits for the context's stream and returns the first device-side status
 * (DBA_ERR_NONFINITE, DBA_ERR_TIMEOUT) or a CUDA error. */
int dba_sync(dba_ctx* ctx);

/* Replaces the host reads of the reference's unified-memory fields (the VTK
 * writers and Integral read them directly): copies field `field` as FP64 into
 * host[nx*ny*nz].  Field ids: dendrite 0 p, 1 T; Model B 0 x, 1 y, 2 z, 3 b,
 * 4 mu_x, 5 mu_y, 6 mu_z; KH 0 Mass, 1 Momx, 2 Momy, 3 Energy, 4 rho, 5 p,
 * 6 vx, 7 vy (primitives recomputed from the conserved fields). */
int dba_read_field(dba_ctx* ctx, int field, double* host);
/* dba_read_field into an FP32 host array of nx*ny*nz values (no counterpart in the
 * reference): the values dba_read_field returns, rounded to float.  For the state fields of
 * an FP32 context this moves half the bytes over the host link. */
int dba_read_field_f32(dba_ctx* ctx, int field, float* host);

/* Replaces the host reads of wake_up / wake_up_next (Output_wakeup,
 * example_Dendritic_growth/kernel.cu:711-757): which = 2*channel + 0 for the
 * wake flags of the next step, 2*channel + 1 for the *_next flags the last
 * step produced.  host[nb] receives 0/1. */
int dba_read_flags(dba_ctx* ctx, int which, int32_t* host);

/* Replaces Calc_RealTime_Values / growth_front / Integral / Calc_Vy_mode
 * (example_Dendritic_growth/kernel.cu:759-863, example_Reactive_ModelB/kernel.cu:920-1010,
 * example_Kelvin_Helmholtz/KH_DBA.cu:1273-1327). */
int dba_observables(dba_ctx* ctx, dba_obs* obs);

/* Replaces growth_front at x = Nx/2 (example_Dendritic_growth/kernel.cu:759-773)
 * alone: gathers one column on the device, cheap enough to poll every few
 * steps.  Dendrite only. */
int dba_tip(dba_ctx* ctx, double* tip);

/* Replaces Output_vtk / write_output_vtk (example_Dendritic_growth/kernel.cu:637-707,
 * example_Reactive_ModelB/kernel.cu:766-879, example_Kelvin_Helmholtz/KH_DBA.cu:1132-1202):
 * ASCII legacy VTK, the reference's header and value formatting. */
int dba_write_vtk(dba_ctx* ctx, const char* path);

/* Replaces Output_wakeup (example_Dendritic_growth/kernel.cu:711-757,
 * example_Reactive_ModelB/kernel.cu:882-917, example_Kelvin_Helmholtz/KH_DBA.cu:1205-1240). */
int dba_write_active_vtk(dba_ctx* ctx, const char* path);

/* No reference counterpart (the reference has no checkpoint): binary
 * snapshot of every state field, flag, parity bit and counter; restoring and
 * stepping is bit-identical to not having stopped. */
int dba_checkpoint(dba_ctx* ctx, const char* path);
int dba_restore(dba_ctx* ctx, const char* path);

int dba_get_info(dba_ctx* ctx, dba_info* info);

/* Copy of the configuration the context was created with. */
int dba_get_config(dba_ctx* ctx, dba_config* cfg);

/* per-kernel device time of profiled steps (dba_step_profiled) */
typedef struct dba_prof {
    int steps;                 /* steps profiled */
    double step_ms;            /* device time of all profiled steps */
    double stencil_ms;         /* device time in the stencil kernel(s): the fused step kernel, or KH's four stages */
    double reduce_ms;          /* conserved-change reduction */
    double correct_ms;         /* conserved correction */
    long active_blocks;        /* block-steps processed (active in any channel) */
    long active_blocks_ch[2];  /* per channel */
    long ch0_only_blocks;      /* dendrite: p-active but not T-active block-steps */
    long cells_per_block;
} dba_prof;

/* No reference counterpart (the reference brackets each kernel with
 * cudaEventRecord/cudaEventSynchronize, example_Dendritic_growth/kernel.cu:919-986):
 * runs nsteps steps without graph capture, with CUDA events around each kernel
 * class on the context's stream, and returns the device times. */
int dba_step_profiled(dba_ctx* ctx, int nsteps, int mode, dba_prof* out);

/* The context's CUDA stream (cudaStream_t), for callers that time or order work on it. */
int dba_get_stream(dba_ctx* ctx, void** stream);

/* No reference counterpart: the checkpoint as an in-memory blob.  dba_save_state
 * copies device state into host[size] (size from dba_state_size), dba_load_state
 * copies it back; both are asynchronous on the context's stream when host is
 * pinned memory and complete before returning otherwise. */
int dba_state_size(dba_ctx* ctx, size_t* size);
int dba_save_state(dba_ctx* ctx, void* host, size_t size);
int dba_load_state(dba_ctx* ctx, const void* host, size_t size);

/* ---- batched simulations (no reference counterpart: the reference runs one
 * simulation per process; these advance many independent 2-D dendrite runs of
 * different sizes and parameters, e.g. an undercooling/anisotropy sweep, with
 * one kernel launch per step over all of their active blocks) ---- */
typedef struct dba_batch dba_batch;

typedef struct dba_batch_config {
    int precision;             /* DBA_PREC_* for every slot */
    int block;                 /* DBA block edge for every slot (4, 8 or 16) */
    int max_slots;             /* simulations held at once */
    int block_capacity;        /* total DBA blocks over all slots */
    size_t cell_capacity;      /* total cells over all slots; 0 = size from free device memory */
    int threads;               /* threads per CTA of the batch kernel: 128, 256 or 512 (0 = 256) */
} dba_batch_config;

typedef struct dba_batch_info {
    size_t free_cells, largest_free_cells;
    long free_blocks, largest_free_blocks;
    int live_slots;
    long step;                 /* batch steps since creation */
    long active_block_steps;   /* blocks processed, summed over steps */
    int grid_ctas;
} dba_batch_info;

int dba_batch_create(const dba_batch_config* cfg, dba_batch** out);
/* Admit one simulation (dendrite, 2-D, cfg->block and cfg->precision equal to
 * the batch's): allocates its fields from the batch arena and its blocks from
 * the block space; DBA_ERR_NOMEM when either has no room.  ic as dba_init. */
int dba_batch_add(dba_batch* b, const dba_config* cfg, const double* ic, int* slot);
int dba_batch_remove(dba_batch* b, int slot);
/* nsteps DBA steps of every live slot (asynchronous; captured graphs). */
int dba_batch_step(dba_batch* b, int nsteps);
int dba_batch_sync(dba_batch* b);
/* growth_front at x = Nx/2 of every slot (NaN for empty slots) and each slot's
 * steps since admission (-1 for empty slots); arrays of max_slots. */
int dba_batch_tips(dba_batch* b, double* tips, long* steps);
int dba_batch_read_field(dba_batch* b, int slot, int field, double* host);
int dba_batch_get_info(dba_batch* b, dba_batch_info* info);
int dba_batch_get_stream(dba_batch* b, void** stream);
void dba_batch_destroy(dba_batch* b);

/* Batch options (no counterpart in the reference).
 *   DBA_BATCH_PERSISTENT  1 (default): dba_batch_step advances its steps in persistent
 *                         launches -- one cooperative launch of up to 48 steps, all CTAs
 *                         resident, a grid barrier between steps; 0: one launch per step.
 *                         Both give the same fields, bit for bit.
 *   DBA_BATCH_WAIT_LIMIT  polls a CTA makes at one grid barrier before it gives up (default
 *                         1 << 24, about a second): the launch then ends early, dba_batch_sync
 *                         returns DBA_ERR_TIMEOUT and the slots' fields are undefined (remove
 *                         and re-add them).  0 gives up at once (a test of the error path).
 * Changing an option waits for the batch's stream and drops its captured graphs. */
#define DBA_BATCH_PERSISTENT 1
#define DBA_BATCH_WAIT_LIMIT 2
int dba_batch_set_option(dba_batch* b, int option, long long value);

/* ---- VTK XML RectilinearGrid output (the reference's CUDA-MPI write_output_vtr /
   write_output_pvtr, example_Dendritic_growth/CUDA-MPI/dendrite_kernels.cu:875-1060) ----
   Writes <base>.vtr, or with pieces > 1 <base>_<r>.vtr for r < pieces (y slabs that
   share their boundary row) and the index <base>.pvtr.  Fields as Float32 (dendrite
   phi, T; Model B X, Y, Z, B; KH rho, p, vx, vy) and the next step's activity per
   cell as Int8 (active_phi / active_T, or active).  DBA_VTR_BINARY: appended raw
   data instead of ASCII.  DBA_VTR_ASYNC: the fields are read now and the files are
   formatted and written by a background thread; dba_wait_io joins the context's
   writers and returns the first write error (dba_destroy waits too). */
#define DBA_VTR_BINARY 1
#define DBA_VTR_ASYNC 2
int dba_write_vtr(dba_ctx* ctx, const char* base, int pieces, int flags);
int dba_wait_io(dba_ctx* ctx);

/* ---- on-device post-processing (the reference's separate analysis tools, run on
   the resident field instead of re-reading ASCII VTK files) ---- */

/* Extract_Tip (example_Dendritic_growth/Extract_Tip.cpp:68-87) on state field `field`:
   for z = Nz/2 + k, k = 0..dz, tip_x[k] = the largest x with value > 0.5 in plane z
   (0 if none, or if the plane is beyond the grid); *tip_x_max = max over k.  The
   tool's Tip_Profile.dat column is tip_x_max - tip_x[k]. */
int dba_tip_profile(dba_ctx* ctx, int field, int dz, int* tip_x, int* tip_x_max);

/* coarsening_analysis (example_Reactive_ModelB/coarsening_analysis.cpp:46-165) of state
   field `field`: avg = (max(0.5, max f) + min(0.5, min f)) / 2; *volume = cells with
   f > avg; islands = periodic 6-connected components grown from cells with f > avg
   through cells with f >= avg; sizes[k] = cells of island k, islands ordered by their
   first f > avg cell in x-fastest order (the tool's scan order).  max_sizes = 0 only
   counts; returns DBA_ERR_ARG (with *islands set) when max_sizes is too small, and
   DBA_ERR_TIMEOUT through dba_sync if the bounded union loop ever gives up. */
int dba_size_distribution(dba_ctx* ctx, int field, double* avg, long* volume, long* islands, long* sizes,
                          long max_sizes);

/* ---- one 2-D domain split into y-slabs across contexts (one per GPU) ----
   The reference's CUDA-MPI programs (example_Dendritic_growth/CUDA-MPI/dendrite.cpp:387-397,
   459-644; example_Reactive_ModelB/CUDA-MPI/reaction.cpp:416-438, 529-552) split the domain
   across ranks and exchange halo layers and wake flags each step.  Here each rank's context
   holds its slab plus one ghost block row on each side (dba_b200/slabs.py drives the
   exchange over torch.distributed).  Dendrite and Model B (2-D).  The calls are
   asynchronous on the context's stream, take device pointers and work between steps.
     dba_rows_pack   current values of rows [row0, row0 + nrows) -> dev_out, field after
                     field (nrows * nx values of the context's precision each): dendrite p, T;
                     Model B x, y, z, then the persisted potentials of x, y, z
     dba_rows_unpack the same layout from dev_in into both buffers of those rows
     dba_flag_rows   the next step's wake flags of block rows [brow0, brow0 + nbrows), every
                     channel (dendrite p then T; nbrows * nbx bytes each): op 0 copies them to
                     dev_buf, op 1 ORs dev_buf into them, op 2 clears them (dev_buf unused),
                     op 3 sets them from dev_buf
     dba_slab_rows   Model B: block rows [first_block_row, first_block_row + block_rows) are
                     this context's own, the others ghosts (never updated, tested or woken
                     from; their flags only say whether their potentials are recomputed or
                     read persisted); domain_cells is the whole domain's cell count, the
                     divisor of the FP32 conserved offset.  Not for FP64 conserved contexts
                     (DBA_ERR_CONFIG: their correction sums per-block values in a fixed tree
                     over one context's blocks).
     dba_lazy_change FP32 conserved Model B: the fixed-point change totals (3 int64, 2^-40
                     units) the last step added, copied to buf (op 0) or replaced from buf
                     (op 1), host or device memory; the slab run sums them over the ranks
                     before the next step. */
int dba_rows_pack(dba_ctx* ctx, int row0, int nrows, void* dev_out);
int dba_rows_unpack(dba_ctx* ctx, int row0, int nrows, const void* dev_in);
int dba_flag_rows(dba_ctx* ctx, int op, int brow0, int nbrows, void* dev_buf);
int dba_slab_rows(dba_ctx* ctx, int first_block_row, int block_rows, long long domain_cells);
int dba_lazy_change(dba_ctx* ctx, int op, void* buf);

/* Context options (no counterpart in the reference).
 *   DBA_OPT_WAIT_LIMIT  attempts a bounded device retry loop makes before it gives up
 *                       (default 1 << 20): the union step of dba_size_distribution, whose
 *                       compare-and-swap retries end with DBA_ERR_TIMEOUT through dba_sync.
 *                       0 gives up at once (a test of the error path). */
#define DBA_OPT_WAIT_LIMIT 1
int dba_set_option(dba_ctx* ctx, int option, long long value);

/* No counterpart in the reference.  For callers that cannot call cudaMalloc
 * -- work enqueued while a stream is captured into a CUDA graph, latency-critical
 * loops that must not take an allocation's implicit device synchronisation, or
 * hosts whose device memory belongs to another allocator: the conserved-DBA
 * mean change, computed with the same fixed-order reduction dba_step uses,
 * allocating nothing.  Its scratch is a fixed array inside the library
 * (32 KiB + 256 B on every GPU that loads it, held until exit).
 *   block_sums: device pointer, nfields x nb FP64 per-block sums of the change
 *   mean_out:   device pointer, nfields FP64 results: sum / ncells
 *   stream:     cudaStream_t to enqueue on (NULL = legacy default stream)
 * Limits: nb <= DBA_NOALLOC_MAX_BLOCKS, 1 <= nfields <= DBA_NOALLOC_MAX_FIELDS;
 * larger sizes return DBA_ERR_ARG.  The first call on a device looks up the
 * array's device address (make it before any stream capture); that address is
 * cached per device index for the life of the process, so it belongs to the
 * device's primary context and does not survive cudaDeviceReset.  All calls share
 * the array: calls that overlap on the GPU race.  Asynchronous on `stream`. */
#define DBA_NOALLOC_MAX_BLOCKS (1 << 20)
#define DBA_NOALLOC_MAX_FIELDS 4
int dba_mean_change_noalloc(const double* block_sums, int nb, int nfields, double ncells, double* mean_out,
                            void* stream);

/* Replaces FreeMemory (example_Dendritic_growth/kernel.cu:866-879). */
void dba_destroy(dba_ctx* ctx);

const char* dba_strerror(int status);

/* sizeof(dba_config), sizeof(dba_obs), sizeof(dba_info): lets a binding check its struct layout. */
size_t dba_struct_size(int which);

#ifdef __cplusplus
}
#endif
#endif /* DBA_H */
