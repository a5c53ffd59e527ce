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
    GF_FIELD_STRAIN_STATIC = 18,      /* static strain, crystal frame (cell, 6)
                                         exxt0_crt..; present with strain_stat.in
                                         or gf_set_elastostatics */
    GF_FIELD_EIGENSTRAIN_STATIC = 19, /* static eigenstrain, crystal frame (cell, 6)
                                         exx0t0_crt..; present with
                                         eigenstraint0_crt.in or gf_set_elastostatics */
    GF_FIELD_FORCE_STORE = 20,        /* stiffness-damping force store (cell, 3)
                                         force_x_store..; elastodynamics */
    GF_FIELD_JP1 = 21,                /* Drude pole currents (cell, 3)  Jpx_n1.. */
    GF_FIELD_JP2 = 22,
    GF_FIELD_JP3 = 23,
    GF_FIELD_COUNT = 24
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
 * H?_Yee.in, elastoforce.in, Jp1-3.in, strain_stat.in, eigenstraint0_crt.in,
 * Hext.in, Eext.in, struct.in).  Replaces the reference's set-up
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

/* ---- Set-up from the host's parsed values -------------------------------
 * For a host that keeps the reference's own readers (read_global,
 * read_materials and set_global, read.cpp:4-237, global.cpp:14-441) and hands
 * the engine what they produced instead of a deck directory.  The names
 * follow global_parameters (global.h:25-176) and material (material.h:3-58).
 * Restart inputs (m.in, p.in, ...) come afterwards through gf_upload, the
 * prescribed H / E tables through gf_set_table. */
typedef struct gf_material_params {
    /* as read from materials.in (read.cpp:121-205), before check_material
     * and get_cijkl: the engine derives B1, B2, F*, tv*, the rotated
     * stiffness and the Drude weights' normalisation the same way */
    double c11, c12, c44, density, elast_mass_damping, elast_stiff_damping;
    int32_t if_FM;
    double Ms, gyro, FM_damping;
    int32_t anisotropy_type;
    double K1, K2, Aex, iDMI, lamda100, lamda111;
    int32_t if_AFM;
    double Ms_AFM[2], gyro_AFM[2], damping_AFM[2], K1_AFM[2], uniaxis_AFM[3], Aex_AFM[2], J_AFM;
    double lamda100_AFM[2], lamda111_AFM[2];
    int32_t if_spin_pump;
    double spin_hall_angle, spin_mix_cond, spin_diffus_length;
    int32_t if_FE;
    double FE_mass, FE_damping, a1, a11, a12, a111, a112, a123, a1111, a1112, a1122, a1123;
    double G11, Q11, Q12, Q44, f11, f12, f44;
    int32_t if_PEC;
    double r_permittivity, conductivity;
    double comp_n[3], omega_plasma_n[3], tao_e_n[3];
} gf_material_params;

typedef struct gf_run_params {
    /* geometry (geometry.h; readgeo, read.cpp:217-237) */
    int64_t nx, ny, nz;
    double dx, dy, dz;
    int32_t periodicX, periodicY, periodicZ;
    /* time stepping and orientation */
    uint64_t step;
    double dt;
    int32_t if_OrientRotate;
    double Tg2c[3][3];             /* Tc2g is its transpose */
    /* uniform initial state of the deck (restart files replace it) */
    double theta_mag, phi_mag, px_init, py_init, pz_init;
    /* external fields */
    double Hext_stat[3], Hext_altr[3], H_altr_freq[3];
    int32_t if_prescribe_Hext;     /* table through gf_set_table(GF_TABLE_HEXT) */
    double Eext_stat[3], Eext_altr[3], E_altr_freq[3];
    int32_t if_prescribe_Eext;     /* table through gf_set_table(GF_TABLE_EEXT) */
    /* magnetostatics / electrostatics */
    int32_t if_magnetostatics, if_mag_1Dmodel, if_demag_factor;
    double demag_fac[3];           /* as read; the engine normalises them to sum -1 */
    int32_t if_elec_1Dmodel, if_elec_1D_compensate;
    double scale_elec; int32_t elec_solver_limit; double elec_solver_tol;
    /* Maxwell */
    int32_t if_EMdynamic, if_input_planeEM_E;
    double planeEM_E[3], planeEM_E_freq[3];
    int32_t if_EM_fromP, if_EM_fromM, if_EM_backaction_on_P, if_EM_backaction_on_M;
    int32_t if_1D_ABC, if_1D_ABC_ELAST_onlytop, if_1D_ABC_EM_onlytop;
    double weighting_factor_fourth_Liao;
    int32_t if_PEC_XY, if_PEC_Z;
    int32_t if_Jf_input;
    int64_t Jfin_lo[3], Jfin_hi[3];   /* Jfin_xi.. and Jfin_xf.. (0-based, inclusive) */
    int32_t Jf_input_type; char Jf_input_component; char pad_[3];
    double Jf_input_amp, Jf_input_freq, Jf_input_sigma; uint64_t num_Jf_cycles;
    /* elastodynamics */
    int32_t if_elastodynamics, if_elasto_backaction_from_pORm, if_elasto_on_pORm;
    int32_t if_gaussian_strain_pulse, input_strain_type, input_strain_sourcez;
    char input_strain_component; char pad2_[7];
    double sigma_gauss, amplitude_gauss; uint64_t num_strain_cycles;
    /* static strain coupling, flexoelectricity, spin pumping; the
     * prescribed-m test mode is not provided (if_prescribed_m must be 0) */
    int32_t if_elastostatic, if_flexo, if_prescribed_m;
    int32_t if_spin_pumping;
    /* elastostatic solve (read.cpp:64; gf_set_elastostatics) */
    double scale_elasto; int32_t elasto_solver_limit; double elasto_solver_tol;
} gf_run_params;

/* Create an engine from the parsed values: `run`, `n_materials` materials and
 * the per-cell material id of set_global (material_cell, nx*ny*nz values in
 * matrix3d order, 0 = vacuum, id-1 indexes `mats`; global.cpp:65-83).
 * Replaces the same set-up sequence as gf_create_from_deck (main.cpp:21-167)
 * with the reading left to the host; the engine reads no file.  An engine
 * made this way from the values a deck holds equals, bit for bit, the one
 * gf_create_from_deck makes from that deck. */
int gf_create(const gf_run_params* run, const gf_material_params* mats, int n_materials, const uint32_t* material_cell,
              int device, int precision, gf_engine** out);

/* Prescribed external-field tables (global.h:52-57, 68-73; read from Hext.in
 * / Eext.in by read_prescribe_Hext / read_prescribe_Eext): n rows of time and
 * x, y, z components.  The table is stepped as the reference does
 * (time_marching_device_serial, global.cpp:512-549): the row index advances
 * when t - dt passes the row's time, and the value is held for the four
 * stages of a step.  The run must have been created with the table switched
 * on (if_prescribe_Hext / if_prescribe_Eext); a new table takes effect from
 * the next step. */
#define GF_TABLE_HEXT 0
#define GF_TABLE_EEXT 1
int gf_set_table(gf_engine* e, int table, const double* times, const double* xyz3, int64_t n);

/* ---- Stage-level stepping ------------------------------------------------
 * For a host that keeps main.cpp's loop and the system classes' method
 * calls: each system's get_d*_RK{s} calls gf_stage_begin(e, s) and its
 * update_*_RK{s} (update_* for s = 4) calls gf_stage_commit(e, s).  The
 * first commit of stage s launches the fused stage of every active physics
 * (the reference's per-system calls of that stage are served by it); further
 * commits of the same stage do nothing, so the call order of main.cpp:252-296
 * (and its repetition for RK2..RK4) works unchanged.  Stages must come in
 * the order 1, 2, 3, 4; the commit of stage 4 completes the step
 * (time_marching_device_serial, the step counter).  Static solves between
 * stages run inside the stage, as in gf_advance; gf_static_solve is for the
 * set-up calls.  Mixing with gf_advance is allowed between whole steps. */
int gf_stage_begin(gf_engine* e, int stage);
int gf_stage_commit(gf_engine* e, int stage);

/* Static field of the current state now: GF_STATIC_MAGNETIC recomputes the
 * magnetostatic field from m (magnetic_system::get_H_static,
 * magnetostatic_solver.cpp:114-219; main.cpp:135-146); GF_STATIC_ELECTRIC
 * runs the electrostatic solve of gf_set_electrostatics, and does nothing
 * while that is off (E_stat stays as it is, as in a build of the reference's
 * public sources, which declare get_E_static without defining it).
 * After a gf_stage_commit (the calls main.cpp makes between stages,
 * main.cpp:299-306, and after a step) it does nothing: the committed stage
 * has already formed the static field of its new state.  Synchronous. */
#define GF_STATIC_MAGNETIC 0
#define GF_STATIC_ELECTRIC 1
int gf_static_solve(gf_engine* e, int which);

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
 * dims of one component; count = 3 * dims product, 6 for the strain fields). */
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
 * *iterations_used (optional) gets the set-up iteration count.
 * With if_elec_1Dmodel the 1-D model replaces the spectral solve
 * (ferroelectric_system::get_E_static_1D, ferroelectric_system.h:106, also
 * undefined in the public sources): the laterally uniform limit of the same
 * periodic electrostatics, per (i, j) column E_z = -(P'_z - D) / (e0 er),
 * D = sum(P'_z / er) / sum(1 / er) (zero mean E_z), E_x = E_y = 0, with
 * P'_z = P_z - P_z(at enabling) under if_elec_1D_compensate; both
 * precisions. */
int gf_set_electrostatics(gf_engine* e, int enable, int* iterations_used);

/* Elastostatic solve: the static strain exxt0_crt of the current static
 * eigenstrain exx0t0_crt (magnetostriction and electrostriction of the
 * current m and p, crystal frame).  Replaces elastic_system::get_strain_static
 * / get_eigenstrain_static (elastic_system.h:184-199), which the reference
 * declares and calls at set-up with elastodynamics and after every step
 * without it (main.cpp:148-156, 213-215, 472-474) but does not define in its
 * public sources; a build of those sources, like the oracle, keeps both at
 * zero (or at strain_stat.in / eigenstraint0_crt.in), and so does the engine
 * until this is enabled.  The solve restates the method the reference's
 * data imply: Khachaturyan's iteration for an elastically inhomogeneous
 * periodic body with the homogeneous cubic stiffness C_h = max(c11, c12,
 * c44) x scale_elasto and its Green tensor (elastic_initialize.cpp:21-40,
 * 340-389), up to elasto_solver_limit iterations or elasto_solver_tol
 * (read.cpp:64), in the crystal frame, with zero mean strain (a clamped
 * box; vacuum layers let a film relax along their normal).  The results act
 * as the reference's static fields do: the LLG adds the static strain to the
 * dynamic one, the dynamic eigenstrain of the elastic and ferroelectric
 * solvers subtracts the static eigenstrain, and with if_elastostatic the
 * ferroelectric field adds both (ferroelectric_solver.cpp:638-651).
 * Enabling solves once now and, without elastodynamics, again after every
 * step with elasto_solver_limit iterations started from the last solution.
 * Decks with flexoelectricity are refused (their static-strain gradients,
 * get_strain_static_glb_gradient, are not built).  Both precisions (the
 * solve itself runs in FP64); *iterations_used (optional) gets the set-up
 * iteration count. */
int gf_set_elastostatics(gf_engine* e, int enable, int* iterations_used);

/* The reference's text outputs (inoutput.cpp:330-887) into directory dir,
 * for the engine's current step nstep (steps done): with initial != 0 the
 * step-0 block of main.cpp:170-198 (averages, Estat, Hstat, strain_stat
 * with elastodynamics, eigenstraint0_crt), otherwise every output whose
 * deck switch (if_output_*) is on and whose interval divides nstep, as
 * main.cpp:486-705 writes them after a step.  Same file names
 * ("m.<nstep>.dat", "Ex_Yee.<nstep>.dat", ...), row order (i, j, k,
 * 1-based), columns and %.7e format; average_*.dat and EM_onecell.dat are
 * appended to.  Fields a run lacks are written as zeros, as the
 * reference's zero-initialised arrays would be.  J_ISHE.<nstep>.dat is not
 * written: the engine forms the inverse-spin-Hall current inside the Yee
 * update and keeps no array of it.  Synchronous. */
int gf_write_outputs(gf_engine* e, const char* dir, int initial);

/* The reference's run in one call (main.cpp:170-705): the step-0 outputs,
 * then the deck's step count from the current step, stopping at every step
 * where an output is due and writing it with gf_write_outputs.  No
 * counterpart besides main.cpp itself. */
int gf_run_deck(gf_engine* e, const char* dir);

/* Full-precision checkpoint of everything that carries from one step to the
 * next: the state fields (and, in the mixed form, their compensation words),
 * the static fields (with the static strain and eigenstrain and the
 * elastostatic solver's iterate), the stage-1 force of the stiffness
 * damping, the Liao boundary history, the step counter and the
 * external-field clock.  A run
 * restarted from it continues bit for bit.  The reference restarts from
 * its %.7e text dumps (inoutput.cpp:330-887, input_* readers); this binary
 * form has no counterpart there.  Load needs an engine created from the same
 * deck and precision (and with the elastostatic solve enabled if it was on
 * in the saved run).  Load reads and checks the whole file before it
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
 * Many engines (uneven grids, either precision) advanced together by one
 * CUDA graph per step parity, in one of three modes:
 *  - phases (GF_BATCH_PHASES): mixed-form engines with TDGL, elastodynamics
 *    and FDTD (Mur boundaries; no magnetism, flexoelectricity, static
 *    solves, plane sources, conductors or Drude poles).  Each RK stage is a
 *    few launches for all engines together — A: elastic tiles, Yee update
 *    and TDGL; B: elastic RK update and the first Mur face direction; C:
 *    elastic boundary planes and the second; D: the third — over lists of
 *    work items (engine, kernel, block), so small grids share the GPU inside
 *    one launch; the launch count per step does not grow with the engine
 *    count (13 for periodic-in-x-and-y decks).  With autotune != 0 the batch
 *    times phase A of stage 1 (which touches no state) for the elastic
 *    tile's x-chunk per item (one chunk for all engines or each engine's
 *    own) and for phase A fused into one launch or split into three
 *    concurrent launches (tile, Yee and TDGL items), and keeps the fastest;
 *    gf_batch_plan describes the choice.
 *  - persistent (GF_BATCH_PERSISTENT): the engines of the phase mode, the
 *    whole step as one cooperative launch (every block resident) over the
 *    same work lists, the phases separated by grid-wide barriers instead of
 *    launches; a barrier that waits too long sets an error that
 *    gf_check_finite of the first engine reports, and the launch returns.
 *  - branches (GF_BATCH_BRANCHES): any engines; each engine's RK4 step is
 *    one branch of the graph.  With autotune != 0 the batch first picks, per
 *    engine, the x-chunk of the tiled elastic kernel by timing it.
 * GF_BATCH_AUTO: branches when some engine does not allow the phase mode;
 * otherwise, with autotune != 0, the fastest of phases, persistent and
 * branches over timed steps whose state is then undone (without autotune,
 * phases).
 * Chunking does not change results.  The engines stay owned by the caller
 * and must not be advanced by other calls while the batch lives; all must
 * sit at steps of the same parity.  The reference runs one system per
 * process; these entry points have no counterpart there. */
typedef struct gf_batch gf_batch;
#define GF_BATCH_AUTO 0
#define GF_BATCH_BRANCHES 1
#define GF_BATCH_PHASES 2
#define GF_BATCH_PERSISTENT 3
int gf_batch_create(gf_engine* const* engines, int count, int autotune, gf_batch** out);   /* GF_BATCH_AUTO */
int gf_batch_create_ex(gf_engine* const* engines, int count, int autotune, int mode, gf_batch** out);
/* Advance every engine by nsteps (asynchronous on the batch stream). */
int gf_batch_advance(gf_batch* b, uint64_t nsteps);
int gf_batch_synchronize(gf_batch* b);
/* The batch's CUDA stream (a cudaStream_t). */
void* gf_batch_stream(gf_batch* b);
/* Elastic-tile x-chunk engine `index` runs with (-1: bad index). */
int gf_batch_tuned_chunk(const gf_batch* b, int index);
/* The batch's mode and tuning choices, as text (valid while b lives). */
const char* gf_batch_plan(const gf_batch* b);
/* Message of the last failing batch call (or failed create when b is NULL). */
const char* gf_batch_last_error(const gf_batch* b);
/* Free the batch (not the engines). */
void gf_batch_destroy(gf_batch* b);

/* ---- Discrete adjoint of the ferromagnetic (magnetoelastic) RK4 step -----
 * Gradients of a loss of the <m_x>(t) trace with respect to an x-directed
 * excitation waveform (n_wave samples, piecewise constant over equal shares
 * of the run, added to the deck's external field) and to a per-cell damping
 * alpha (new inputs: the reference has per-material alpha only,
 * magnetic_solver.cpp:206).  Differentiates the engine's discretisation of
 * get_dm_RK{1..4} / update_m_RK* / update_m (magnetic_solver.cpp:3-229,
 * 1515-1636) with per-stage FFT magnetostatics (magnetostatic_solver.cpp:
 * 114-219): exchange, anisotropy (no frame rotation), Zeeman; and, on decks
 * with elastodynamics, the magnetoelastic field of the cell strain
 * (magnetic_solver.cpp:148-156), the stress divergence with the
 * magnetostrictive eigenstrain and the elastic RK4 with step-start mass
 * damping and the stiffness-damping force store (elastic_dynamic_solver.cpp:
 * 3-104, 841-1329, 2801-3057) and the Liao boundary at k = 0
 * (elastodynamics_AbsorbingBoundary.cpp:91-230), whose history reaches
 * three steps back.  Decks with DMI, AFM, FE or Maxwell fields, the Mur
 * elastic boundary (if_1D_ABC), an elastic source, static strain inputs,
 * ny < nz (the reference's z-face neighbour rule for k = ny-1) or nz < 5
 * are GF_EUNSUPPORTED.  The reference has no adjoint; these entry points
 * have no counterpart there.  On an FP64 engine the adjoint computes in
 * FP64; on a mixed-form engine its forward run, stage fields and cotangents
 * are FP32 (step values with compensation words, the engine's own FP32
 * elastic kernels and FFT path; |m| is not renormalised) while the damping
 * and waveform gradients, the <m_x> trace and its cotangent stay FP64.  The
 * adjoint uses the engine's stream and FFT buffers: do not advance the
 * engine while an adjoint call runs. */
typedef struct gf_adjoint gf_adjoint;
/* checkpoint_every: steps between stored states (the backward run recomputes
 * the steps in between).  Device memory: a stored state is 24 * n bytes, 96
 * with elastodynamics (mixed form 24 and 84) per checkpoint; the backward run
 * adds one block's stage store, checkpoint_every * 192 * n bytes (384 with
 * the magnetoelastic field; half in the mixed form), when it fits (see
 * gf_adjoint_set_store_limit), else one block's step values (the stored
 * state's size per step) and a second forward evaluation of every step. */
int gf_adjoint_create(gf_engine* e, int n_wave, int checkpoint_every, gf_adjoint** out);
/* per-cell damping (nx*ny*nz values; default: the material's alpha) */
int gf_adjoint_set_alpha(gf_adjoint* a, const double* alpha, size_t count);
/* waveform samples in A/m (n_wave values; default 0) */
int gf_adjoint_set_waveform(gf_adjoint* a, const double* w, size_t count);
/* Run nsteps RK4 steps from the engine's current state (m; with
 * elastodynamics also u, v, the force store and the Liao history) and
 * external-field clock (the engine's own state is not advanced); mx_trace
 * gets <m_x> at steps 0..nsteps (nsteps+1 values). Synchronous. */
int gf_adjoint_forward(gf_adjoint* a, uint64_t nsteps, double* mx_trace);
/* Given dloss/d<m_x> at steps 0..nsteps (nsteps+1 values), the gradients
 * with respect to the waveform (n_wave values) and the per-cell alpha
 * (nx*ny*nz values). Synchronous. */
int gf_adjoint_backward(gf_adjoint* a, const double* dloss_dmx, double* grad_wave, double* grad_alpha);
/* m after the last forward step (3*nx*ny*nz values, component-major). */
int gf_adjoint_final_m(gf_adjoint* a, double* host_m, size_t count);
/* Device memory the backward run may hold for a block's stage store (the
 * stage states, fields and strains of every step of a checkpoint block, so
 * that each step is evaluated once in the reverse pass instead of twice):
 * -1 (default) = when it fits the device's free memory less a reserve of
 * max(4 GiB, 1/16 of the device); 0 = never; > 0 = at most that many bytes.
 * Both layouts give identical gradients. */
int gf_adjoint_set_store_limit(gf_adjoint* a, int64_t bytes);
/* Layout of the last backward run: *used = 1 with the stage store, 0 with
 * the step values only; *bytes = the memory that layout held. */
int gf_adjoint_store_info(gf_adjoint* a, int* used, int64_t* bytes);
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
