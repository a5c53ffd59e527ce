/*
 * goferro_b200.h — C ABI of the B200 engine for GO-Ferro's coupled dynamical
 * phase-field RK4 time step (LLG magnetisation, second-order ferroelectric
 * polarisation dynamics, elastodynamics, Yee-grid Maxwell, FFT
 * magnetostatics).
 *
 * The reference has no plugin API: its boundary is the public methods and
 * fields of four C++ system classes that main.cpp drives
 * (magnetic_system.h:158-211, ferroelectric_system.h:95-132,
 * elastic_system.h:172-225, EMdynamic_system.h:131-180).  Each entry point
 * below replaces a group of those methods; the reference interface it stands
 * in for is cited beside it.  Plain pointers and sizes only; every call
 * returns GF_OK (0) or a negative GF_E* code, and gf_last_error() gives the
 * message.  One engine owns its device memory and CUDA stream; engines are
 * independent and may live on different host threads.
 *
 * Storage order of every field is the reference's matrix3d order
 * (matrix.h:46-52): index = (i*dimy + j)*dimz + k, z fastest, one array per
 * vector component.  Cell fields have dims (nx, ny, nz); the Yee fields have
 * the staggered dims of EMdynamic_initialize.cpp:71-93:
 *   Ex (nx, ny+1, nz+1)  Ey (nx+1, ny, nz+1)  Ez (nx+1, ny+1, nz)
 *   Hx (nx+1, ny, nz)    Hy (nx, ny+1, nz)    Hz (nx, ny, nz+1)
 */
#ifndef GOFERRO_B200_H
#define GOFERRO_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gf_engine gf_engine;

/* status codes */
#define GF_OK 0
#define GF_EINVAL (-1)       /* bad argument or unsupported deck option   */
#define GF_EIO (-2)          /* deck or restart file missing / malformed  */
#define GF_ECUDA (-3)        /* CUDA runtime or cuFFT failure              */
#define GF_ENOMEM (-4)       /* device allocation failed                   */
#define GF_ENAN (-5)         /* non-finite value found by a health check   */
#define GF_ENODEV (-6)       /* no usable sm_100 device                    */
#define GF_EUNSUPPORTED (-7) /* deck asks for physics the engine lacks    */

/* fields for gf_upload / gf_download / gf_field_dims (component-major:
 * a vector field is 3 consecutive arrays x, y, z of the field's dims) */
enum gf_field {
    GF_FIELD_M = 0,       /* FM magnetisation m (cell, 3)       mx_glb..   */
    GF_FIELD_M_AFM1 = 1,  /* AFM sublattice 1 (cell, 3)         mx_AFM1_glb */
    GF_FIELD_M_AFM2 = 2,  /* AFM sublattice 2 (cell, 3)         mx_AFM2_glb */
    GF_FIELD_P = 3,       /* polarisation p (cell, 3)           px_glb..    */
    GF_FIELD_Q = 4,       /* dp/dt (cell, 3)                    qx_glb..    */
    GF_FIELD_U = 5,       /* displacement (cell, 3)             Dux_glb..   */
    GF_FIELD_V = 6,       /* velocity (cell, 3)                 vx_glb..    */
    GF_FIELD_EX = 7,      /* Yee E components, one array each   DEx_em..    */
    GF_FIELD_EY = 8,
    GF_FIELD_EZ = 9,
    GF_FIELD_HX = 10,     /* Yee H components                   DHx_em..    */
    GF_FIELD_HY = 11,
    GF_FIELD_HZ = 12,
    GF_FIELD_HSTAT = 13,  /* magnetostatic field (cell, 3)      Hx_stat..   */
    GF_FIELD_ESTAT = 14,  /* electrostatic field (cell, 3)      Ex_stat..   */
    GF_FIELD_E_CELL = 15, /* cell-centred E (cell, 3), read-only DEx_em_cell */
    GF_FIELD_H_CELL = 16, /* cell-centred H (cell, 3), read-only DHx_em_cell */
    GF_FIELD_STRAIN = 17, /* dynamic cell strain, global frame (cell, 6:
                             xx yy zz yz xz xy), read-only   Dexx_glb..    */
    GF_FIELD_COUNT = 18
};

/* observables for gf_average (global averages, FP64 sums) */
enum gf_obs {
    GF_OBS_M = 0,     /* sum(m)/NFM           magnetic_solver.cpp:1863-1888   */
    GF_OBS_M_AFM1 = 1,/* sum(m1)/NAFM         magnetic_AFM_solver.cpp:2221    */
    GF_OBS_M_AFM2 = 2,/* sum(m2)/NAFM                                          */
    GF_OBS_P = 3,     /* sum(p)/NFE           ferroelectric_solver.cpp:2031   */
    GF_OBS_U = 4      /* sum(u)/n  (mean displacement over all cells)          */
};

typedef struct gf_info {
    int32_t nx, ny, nz;
    double dx, dy, dz;
    double dt;
    double time;            /* physical time reached (time_device)           */
    uint64_t step;          /* completed steps                               */
    uint64_t deck_steps;    /* `step` line of system_setting.in              */
    int32_t n_materials;
    int32_t fm, afm, fe, elastic, em, demag_per_stage; /* active physics     */
    uint64_t n_fm, n_afm, n_fe;  /* NFM, NAFM, NFE (global.cpp:103-118)      */
    uint64_t device_bytes;  /* device memory the engine holds                */
    int32_t launches_per_step;  /* engine kernels launched per RK4 step      */
    int32_t precision;          /* GF_PRECISION_FP64 or GF_PRECISION_MIXED_FP32 */
} gf_info;

/* Accumulated device time of one kernel family (gf_profile_steps). */
typedef struct gf_kernel_time {
    char name[40];
    int32_t launches;
    double total_ms;
} gf_kernel_time;

/* Create an engine from a GO-Ferro input deck directory: system_setting.in,
 * materials.in and whatever restart / table files the deck switches on
 * (m.in, m_AFM.in, Hstat.in, p.in, q.in, Estat.in, u.in, v.in, E?_Yee.in,
 * H?_Yee.in, Hext.in, Eext.in, struct.in).  Replaces the reference's set-up
 * sequence main.cpp:21-167 (readgeo, read_global, *initialize_host,
 * input_*, copy_to_device, initialize_device and the initial static
 * solves).  `device` selects the CUDA device (-1 = current). */
int gf_create_from_deck(const char* deck_dir, int device, gf_engine** out);

/* Arithmetic of an engine (gf_create_from_deck_ex).
 *   GF_PRECISION_FP64: every field, stencil and transform in FP64, evaluated
 *     in the reference's operation order (the parity form).
 *   GF_PRECISION_MIXED_FP32: state arrays, stencils and FFTs in FP32; each
 *     state scalar carries an FP32 compensation word, so the RK4 step value
 *     X + C accumulates increments without FP32 rounding drift; |m| is
 *     renormalised to 1 after every stage (the reference does not
 *     renormalise).  The demag tensor and its spectra are built in FP64; the
 *     averages and every upload/download stay FP64 at this ABI.
 *     Every physics of the FP64 form runs in both; the electrostatic
 *     solve and the adjoint are FP64 only. */
#define GF_PRECISION_FP64 0
#define GF_PRECISION_MIXED_FP32 1

/* gf_create_from_deck with a choice of arithmetic.  Replaces the same set-up
 * sequence (main.cpp:21-167); the reference has only its FP64 build. */
int gf_create_from_deck_ex(const char* deck_dir, int device, int precision, gf_engine** out);

/* Advance `nsteps` full RK4 steps.  Replaces the body of the reference time
 * loop main.cpp:243-484: time_marching_device_serial, the four stages of
 * get_d*_RK{1..4} / update_*_RK{1..3} / update_* for every active system,
 * and the between-stage magnetostatic solves.  Asynchronous on the engine's
 * stream; the step is captured once as a CUDA graph and replayed. */
int gf_advance(gf_engine* e, uint64_t nsteps);

/* Same as gf_advance but launches the kernels directly without a graph
 * (used for debugging and for timing the graph's benefit). */
int gf_advance_eager(gf_engine* e, uint64_t nsteps);

/* Global average of an observable (gf_obs) of the current state, FP64.
 * Replaces get_averagem / get_averagem_AFM / get_averagep. Synchronous. */
int gf_average(gf_engine* e, int obs, double out3[3]);

/* Cell-centred E and H at cell (i,j,k) (0-based), as the reference's
 * output_em_onecell reads them (DE?_em_cell / DH?_em_cell). Synchronous. */
int gf_probe_em(gf_engine* e, int64_t i, int64_t j, int64_t k, double e3[3], double h3[3]);

/* Number of doubles and dims of one array of a field (for vector fields the
 * dims of one component; count = 3 * dims product, 6 for GF_FIELD_STRAIN). */
int gf_field_dims(gf_engine* e, int field, int64_t dims3[3], size_t* count);

/* Copy a field to / from host memory (count doubles, component-major).
 * Replace the reference's copy*_from_device and input_* restart readers.
 * A magnetisation (m, m_AFM1, m_AFM2) uploaded before the first step stands
 * for the restart file read at set-up: the static magnetic field is formed
 * again from it, as the reference computes it before its time loop
 * (main.cpp:135-146), unless the deck supplies Hstat.in.  Synchronous. */
int gf_download(gf_engine* e, int field, double* host, size_t count);
int gf_upload(gf_engine* e, int field, const double* host, size_t count);

/* Same as gf_download but into device memory owned by the caller
 * (cudaMemcpyAsync device-to-device on the engine stream, no host sync). */
int gf_download_device(gf_engine* e, int field, double* dev, size_t count);
/* Same as gf_upload but from caller-owned device memory. */
int gf_upload_device(gf_engine* e, int field, const double* dev, size_t count);

/* Advance `nsteps` steps like gf_advance_eager, with a CUDA event pair
 * around every kernel launch, and report the summed device time per kernel
 * family (at most max_records records; *n_records gets the count).  The
 * state advances exactly as with gf_advance.  Replaces nothing in the
 * reference, which has only a wall-clock stamp around the loop
 * (main.cpp:209-211, 720-726). */
int gf_profile_steps(gf_engine* e, uint64_t nsteps, gf_kernel_time* out, int max_records, int* n_records);

/* Electrostatic (depolarisation) field of the polarisation, E_stat.
 * Replaces ferroelectric_system::get_E_static (ferroelectric_system.h:103),
 * which the reference declares and calls (main.cpp:122-131, 299-302) but does
 * not define in its public sources; a build of those sources, like the
 * oracle, keeps E_stat at zero (or at Estat.in), and so does the engine
 * until this is enabled.  The solve restates the method the reference's data
 * imply: spectral, periodic, with the homogeneous reference permittivity
 * er_h = max(er) * scale_elec (ferroelectric_initialize.cpp:310-338) and a
 * fixed-point iteration for the cells whose er differs from er_h, up to
 * elec_solver_limit iterations or elec_solver_tol (read.cpp:56).  Enabling
 * solves once now (unless Estat.in was read) and, without Maxwell fields,
 * after every RK stage with elec_solver_limit iterations.  FP64 engines;
 * *iterations_used (optional) gets the set-up iteration count. */
int gf_set_electrostatics(gf_engine* e, int enable, int* iterations_used);
/* Full-precision checkpoint of everything that carries from one step to the
 * next: the state fields (and, in the mixed form, their compensation words),
 * the static fields, the stage-1 force of the stiffness damping, the Liao
 * boundary history, the step counter and the external-field clock.  A run
 * restarted from it continues bit for bit.  The reference restarts from
 * its %.7e text dumps (inoutput.cpp:330-887, input_* readers); this binary
 * form has no counterpart there.  Load needs an engine created from the same
 * deck and precision.  Load reads and checks the whole file before it
 * writes any device buffer, so a file that fails (wrong deck, precision,
 * size or a short read) leaves the engine as it was. Synchronous. */
int gf_save_state(gf_engine* e, const char* path);
int gf_load_state(gf_engine* e, const char* path);

/* Engine facts (grid, active physics, counters). */
int gf_get_info(gf_engine* e, gf_info* info);

/* Wait for all work queued on the engine stream. */
int gf_synchronize(gf_engine* e);

/* The engine's CUDA stream (a cudaStream_t), for callers that queue their
 * own work behind the engine. */
void* gf_stream(gf_engine* e);

/* Check every state field for non-finite values on the device; returns
 * GF_ENAN and names the first offending field in gf_last_error. */
int gf_check_finite(gf_engine* e);

/* Message of the last failing call on this engine (or of the last failing
 * gf_create_from_deck when e is NULL).  Never NULL. */
const char* gf_last_error(const gf_engine* e);

/* Free the engine and all its device memory. */
void gf_destroy(gf_engine* e);

/* ---- Batched runs --------------------------------------------------------
 * Many engines (uneven grids, either precision) advanced together: each
 * engine's RK4 step is one branch of a single CUDA graph per step parity, so
 * one graph launch advances every instance and small instances run
 * concurrently.  With autotune != 0 the batch first picks, per engine, the
 * x-chunk of the tiled elastic kernel by timing it (the state is not
 * touched; chunking does not change results).  The engines stay owned by
 * the caller and must not be advanced by other calls while the batch lives;
 * all must sit at steps of the same parity.  The reference runs one system
 * per process; these entry points have no counterpart there. */
typedef struct gf_batch gf_batch;
int gf_batch_create(gf_engine* const* engines, int count, int autotune, gf_batch** out);
/* Advance every engine by nsteps (asynchronous on the batch stream). */
int gf_batch_advance(gf_batch* b, uint64_t nsteps);
int gf_batch_synchronize(gf_batch* b);
/* The batch's CUDA stream (a cudaStream_t). */
void* gf_batch_stream(gf_batch* b);
/* Elastic-tile x-chunk engine `index` runs with (-1: bad index). */
int gf_batch_tuned_chunk(const gf_batch* b, int index);
/* Message of the last failing batch call (or failed create when b is NULL). */
const char* gf_batch_last_error(const gf_batch* b);
/* Free the batch (not the engines). */
void gf_batch_destroy(gf_batch* b);

/* ---- Discrete adjoint of the ferromagnetic RK4 step ---------------------
 * Gradients of a loss of the <m_x>(t) trace with respect to an x-directed
 * excitation waveform (n_wave samples, piecewise constant over equal shares
 * of the run, added to the deck's external field) and to a per-cell damping
 * alpha (new inputs: the reference has per-material alpha only,
 * magnetic_solver.cpp:206).  Differentiates the engine's discretisation of
 * get_dm_RK{1..4} / update_m_RK* / update_m (magnetic_solver.cpp:3-229,
 * 1515-1636) with per-stage FFT magnetostatics (magnetostatic_solver.cpp:
 * 114-219): exchange, anisotropy (no frame rotation), Zeeman; decks with
 * DMI, AFM, FE, elastic or Maxwell fields are GF_EUNSUPPORTED.  The reference
 * has no adjoint; these entry points have no counterpart there.  FP64 engines
 * only.  The adjoint uses the engine's stream and FFT buffers: do not advance
 * the engine while an adjoint call runs. */
typedef struct gf_adjoint gf_adjoint;
/* checkpoint_every: steps between stored states (the backward run recomputes
 * the steps in between; device memory ~ 24 * n * checkpoint_every bytes). */
int gf_adjoint_create(gf_engine* e, int n_wave, int checkpoint_every, gf_adjoint** out);
/* per-cell damping (nx*ny*nz values; default: the material's alpha) */
int gf_adjoint_set_alpha(gf_adjoint* a, const double* alpha, size_t count);
/* waveform samples in A/m (n_wave values; default 0) */
int gf_adjoint_set_waveform(gf_adjoint* a, const double* w, size_t count);
/* Run nsteps RK4 steps from the engine's current m and external-field clock
 * (the engine's own state is not advanced); mx_trace gets <m_x> at steps
 * 0..nsteps (nsteps+1 values). Synchronous. */
int gf_adjoint_forward(gf_adjoint* a, uint64_t nsteps, double* mx_trace);
/* Given dloss/d<m_x> at steps 0..nsteps (nsteps+1 values), the gradients
 * with respect to the waveform (n_wave values) and the per-cell alpha
 * (nx*ny*nz values). Synchronous. */
int gf_adjoint_backward(gf_adjoint* a, const double* dloss_dmx, double* grad_wave, double* grad_alpha);
/* m after the last forward step (3*nx*ny*nz values, component-major). */
int gf_adjoint_final_m(gf_adjoint* a, double* host_m, size_t count);
void gf_adjoint_destroy(gf_adjoint* a);

/* Mean of a device array, allocating nothing: *dev_out = sum(dev_in[0..n)) /
 * divisor, as a deterministic FP64 sum queued on `stream` (a cudaStream_t;
 * NULL = legacy default stream).  No counterpart in the reference.
 *
 * For callers that cannot allocate device memory while they run: code whose
 * device memory belongs to another runtime (the reference's OpenACC data
 * regions, a caller-managed pool), or that runs where cudaMalloc is not
 * allowed or would stall the device (it synchronises the whole device, and
 * it cannot be called while a stream is being captured).  Inputs and output
 * are caller-owned device pointers; the partial sums live in a fixed
 * file-scope device array of 65,600 doubles (about 513 KB) that every GPU
 * which loads the library holds until the process exits.
 *   - n must be 1..67,108,864 (64 Mi); larger inputs return GF_EINVAL with
 *     the limit in gf_last_error(NULL).
 *   - The first call on a device looks up that array's device address; make
 *     that first call before any stream capture on the device.  The address
 *     is kept for the life of the process: after cudaDeviceReset (or any
 *     other end of the device's primary context) the entry point must not be
 *     called again on that device.
 *   - All calls on a device share the array: calls that overlap on the GPU
 *     (two streams, two host threads) race and give wrong sums.  Serialise
 *     them on one stream.
 * Errors are reported through gf_last_error(NULL). */
int gf_field_mean_noalloc(const double* dev_in, uint64_t n, double divisor, double* dev_out, void* stream);

/* Diagnostic: the stencil kernels divide by run constants (cell sizes, dt,
 * the RK4 weights 3 and 6) with a reciprocal-and-correction sequence
 * instead of the general division.  This queues, on the current device,
 * n quotients x / d for pseudo-random x of magnitude 1e-30..1e30 (half of
 * them close to rounding midpoints) with seed `seed`, computes each both
 * ways and stores in *mismatches how many differ in any bit.  No
 * counterpart in the reference; the reference divides with IEEE division,
 * so 0 mismatches means the kernels' quotients equal the reference's. */
int gf_check_quotients(double d, uint64_t n, uint64_t seed, uint64_t* mismatches);

/* Library version string. */
const char* gf_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GOFERRO_B200_H */
