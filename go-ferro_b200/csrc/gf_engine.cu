// B200 engine for GO-Ferro's coupled RK4 phase-field step: state ownership,
// stage sequencing, CUDA-graph replay and the C ABI of goferro_b200.h.
//
// One translation unit holds every kernel (the .cuh files below); it is
// compiled with -fmad=false so that each multiply and add of the FP64 parity
// form is rounded separately, as in the reference's host build.
//
// Two precisions share the engine.  The FP64 form (GF_PRECISION_FP64) is the
// parity path.  The mixed form (GF_PRECISION_MIXED_FP32) instantiates the
// same stage kernels with R = float: state arrays, stencils and transforms
// in FP32, a compensation word per state scalar (gf_state.cuh), |m| = 1 after
// every stage; FP64 remains in the demag-table build, the averages and the
// conversions at this ABI, which takes and returns FP64 in both forms.  The
// device buffers below are held through double* handles in both forms: in
// the mixed form they are allocated at 4 bytes per element and hold FP32
// values, and build_io hands the kernels float* views of them.
#include <cuda_runtime.h>
#include <cufft.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/goferro_b200.h"
#include "gf_deck.h"
#include "gf_launch.cuh"
#include "gf_state.cuh"
#include "gf_elastic.cuh"
#include "gf_llg.cuh"
#include "gf_fe.cuh"
#include "gf_em.cuh"
#include "gf_demag.cuh"
#include "gf_util.cuh"
#include "gf_adjoint.cuh"
#include "gf_batch.cuh"
#include "gf_elec.cuh"
#include "gf_elasto.cuh"

using namespace gf;

struct Field3 {
    // X, A, S0, S1 per component; len[c] = elements of component c
    double* X[3] = {nullptr, nullptr, nullptr};
    double* A[3] = {nullptr, nullptr, nullptr};
    double* S0[3] = {nullptr, nullptr, nullptr};
    double* S1[3] = {nullptr, nullptr, nullptr};
    double* C[3] = {nullptr, nullptr, nullptr};   // compensation words (mixed form only)
    long len[3] = {0, 0, 0};
    bool on = false;
};

namespace {

constexpr int kThreads = 256;
constexpr long kDriveCap = 4096;      // steps of time-dependent drive held on the device (power of two)
thread_local std::string g_create_err;

}  // namespace

struct gf_engine {
    Deck deck;
    Params P{};
    int device = 0;
    bool mixed = false;                    // GF_PRECISION_MIXED_FP32
    size_t esz = sizeof(double);           // bytes per element of the real-valued device buffers
    cudaStream_t stream = nullptr;
    // branch streams of a stage (LLG, TDGL, Maxwell) and their fork / join
    // events; the elastic chain and the static solves stay on `stream`
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    bool prio_nodes = false;               // the streams have unequal priorities (kept by the step graph)
    cudaEvent_t bev[6] = {};
    std::string err;

    // bookkeeping
    std::vector<void*> allocs;
    size_t bytes = 0;
    unsigned long long steps_done = 0;     // completed steps (host mirror of the device counter)
    double t_host = 0.;                    // time_device after the last computed step
    long presc_H = 0, presc_E = 0;
    double Hext_cur[3] = {0, 0, 0}, Eext_cur[3] = {0, 0, 0};

    // device data
    uint8_t* mid = nullptr;
    DevMat* mats = nullptr;
    LLGTables* llg_tab = nullptr;
    DevMatT<float>* mats_f = nullptr;      // mixed form: FP32 copies of the tables
    LLGTablesT<float>* llg_tab_f = nullptr;
    StepDrive* drive = nullptr;
    StepDrive* drive_host = nullptr;       // pinned staging
    unsigned long long* step_ctr = nullptr;
    double* jf_kfac = nullptr;
    double* ishe_coef = nullptr;           // per k (run precision)
    int* ishe_src = nullptr;               // per k
    uint8_t* ecls[3] = {nullptr, nullptr, nullptr};   // material class of every E edge (setup_em_classes)
    void* em_cls_tab = nullptr;            // EmCls<R> table of the run precision
    int em_ncls = 0;

    Field3 m, a1, a2, p, q, u, v, E, H;
    Field3 jp[3];                      // Drude pole currents
    double* dm[3] = {nullptr, nullptr, nullptr};
    double* da1[3] = {nullptr, nullptr, nullptr};
    double* da2[3] = {nullptr, nullptr, nullptr};
    double* force_store[3] = {nullptr, nullptr, nullptr};
    double* force[3] = {nullptr, nullptr, nullptr};
    double* Hstat[3] = {nullptr, nullptr, nullptr};
    double* Estat[3] = {nullptr, nullptr, nullptr};
    double* Hnu[3] = {nullptr, nullptr, nullptr};
    double* fg[9] = {};
    double* strain_c[6] = {};
    double* flexo_sg[6] = {};          // flexoelectric scratch (StageIOT::sg, pge)
    double* flexo_pge[6] = {};
    ETileMaps etm[2][4] = {};          // TMA maps of k_elastic_tile per step parity and stage
    unsigned* tma_err = nullptr;       // set by a timed-out TMA wait
    int el_chunk = 1;                  // x-planes per block of k_elastic_tile
    int el_nmat = 0;                   // materials staged by k_elastic_tile
    size_t el_smem = 0;                // its dynamic shared memory
    bool el_cubic = false;             // every material has the cubic stiffness pattern
    double* liao_hist = nullptr; double* liao_last = nullptr;
    double* scratch = nullptr;             // output staging (scratch_main doubles), then reduction partials
    size_t scratch_main = 0;
    int* flag = nullptr;

    // magnetostatics
    int demag_mode = -1;                   // -1 none, 0 FFT, 1 factors, 2 1-D
    bool demag_per_stage = false;
    bool demag_src_fused = false;          // the LLG kernel writes the transform's input (StageIOT::msrc)
    double* Mfft = nullptr;                // 3 x n real
    cufftDoubleComplex* Mk = nullptr;      // 3 x n21
    cufftDoubleComplex* Nk = nullptr;      // FP64 form: the nine complex demag spectra, 9 x n21
    float* Nr = nullptr;                   // mixed form: the six real spectra, 6 x n21
    cufftHandle plan_r2c = 0, plan_c2r = 0;
    bool plans = false;

    // electrostatic field of P (gf_set_electrostatics; gf_elec.cuh)
    bool elec_on = false, elec_per_stage = false;
    int elec_iters = 1;                    // iterations of each per-stage solve
    double elec_erh = 1.;                  // homogeneous reference permittivity
    double* elec_k[3] = {nullptr, nullptr, nullptr};   // kx (nx), ky (ny), kz (nz/2+1)
    double* elec_q = nullptr;              // 3 x n real
    cufftDoubleComplex* elec_qk = nullptr; // 3 x n21
    double* elec_blockmax = nullptr;       // 2 x kElecBlocks
    cufftHandle elec_r2c = 0, elec_c2r = 0;
    bool elec_plans = false;
    bool elec_1d = false;                  // the 1-D model replaces the spectral solve
    double* elec_pz_t0 = nullptr;          // P_z when the compensated 1-D model was enabled (type R)
    // static strain exxt0_crt and static eigenstrain exx0t0_crt (type R, 6
    // arrays each; null when absent): strain_stat.in / eigenstraint0_crt.in
    // or the elastostatic solve (gf_set_elastostatics)
    double* es_eps[6] = {};
    double* es_eig[6] = {};
    bool es_on = false, es_per_step = false;
    int es_iters = 1;                      // iterations of each per-step solve
    double es_ch[3] = {0., 0., 0.};        // C_h: c11, c12, c44
    EsMats es_mats = {};                   // crystal-frame cubic constants per material
    double* es_x = nullptr;                // 6 x n FP64 strain iterate
    double* es_e0 = nullptr;               // 6 x n FP64 static eigenstrain
    double* es_r = nullptr;                // 6 x n FP64 tau / inverse transform
    cufftDoubleComplex* es_k = nullptr;    // 6 x n21
    double* es_G = nullptr;                // 6 x n21 Green tensor (11 22 33 12 13 23)
    double* es_kq = nullptr;               // 3 x n21 crystal-frame wave vector
    int* es_nyq_idx = nullptr;             // n21: row of es_nyq_op, -1 off the Nyquist planes
    double* es_nyq_op = nullptr;           // 36 per Nyquist point: sign-averaged operator
    double* es_blockmax = nullptr;
    cufftHandle es_r2c = 0, es_c2r = 0;
    bool es_plans = false;

    StageIO io[2][4];
    StageIOT<float> iof[2][4];             // mixed form
    // launch accounting and optional per-launch timing (gf_profile_steps)
    int launches_per_step = 0;
    // stage-level stepping (gf_stage_begin / gf_stage_commit): 0 = no step
    // open, else the stage last committed + 1 (1..4) of the open step
    int stage_open = 0;
    int stage_done = 0;
    int launch_counter = 0;
    bool profiling = false;
    struct ProfRec { const char* name; cudaEvent_t a, b; };
    std::vector<ProfRec> prof;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    bool graphs_ready = false;
};

// The mixed form's stage kernels are instantiated only in gf_mixed.cu, which
// includes this file with GF_MIXED_TU defined and is compiled with FMA
// contraction (the FP64 parity kernels here must not contract).  These two
// functions are its interface.
int gf_mixed_enqueue_step(gf_engine* eng, int parity);                 // kernels of one step, mixed form
int gf_mixed_enqueue_stage(gf_engine* eng, int parity, int s);         // kernels of stage s (0..3), mixed form
int gf_mixed_elastic_setup(gf_engine* eng, int smem, int* per_sm);   // shared-memory opt-in, occupancy
int gf_mixed_time_tile(gf_engine* eng, int reps, float* ms);          // stage-1 elastic tile, mean ms per launch
int gf_mixed_adj_elastic(gf_engine* eng, int s, int rk, const StageIOT<float>& io);  // adjoint: FP32 elastic tile / RK of stage s
int gf_mixed_batch_attr(size_t smem);                                   // shared-memory opt-in of the batch phase kernels
int gf_mixed_batch_persistent_blocks(size_t smem, int* blocks);          // co-resident blocks of k_batch_persistent
int gf_mixed_batch_persistent(const BatchInst* insts, int ninst, const BatchItem* A, int nA, const BatchItem* L, int nB, int nC,
                              int nD, int parity, size_t smem, unsigned* err, unsigned* bar, int blocks, cudaStream_t st);
int gf_mixed_batch_phase(const BatchInst* insts, const BatchItem* items, int count, int s, int ph, int parity, size_t smem,
                         unsigned* tma_err, cudaStream_t st);                 // one phase launch of a batch (a cudaError_t)

namespace {

#define GF_CU(call)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            eng->err = std::string(#call) + ": " + cudaGetErrorString(e_);               \
            return GF_ECUDA;                                                             \
        }                                                                                \
    } while (0)

#define GF_FFT(call)                                                                     \
    do {                                                                                 \
        cufftResult r_ = (call);                                                         \
        if (r_ != CUFFT_SUCCESS) {                                                       \
            eng->err = std::string(#call) + ": cuFFT error " + std::to_string((int)r_);  \
            return GF_ECUDA;                                                             \
        }                                                                                \
    } while (0)

#define GF_TRY(expr)                      \
    do {                                  \
        int rc_ = (expr);                 \
        if (rc_ != GF_OK) return rc_;     \
    } while (0)

cudaEvent_t next_event(gf_engine* eng) {
    if (eng->ev_used == eng->ev_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        eng->ev_pool.push_back(e);
    }
    return eng->ev_pool[eng->ev_used++];
}

// every kernel of the engine is launched through klaunch: it counts the
// launch and, in profiling mode, brackets it with events on the stream
template <bool Tiled = false, class Kernel, class... Args>
cudaError_t klaunch(gf_engine* eng, const char* name, Kernel k, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                    Args... args) {
    cudaEvent_t a = nullptr, b = nullptr;
    if (eng->profiling) { a = next_event(eng); cudaEventRecord(a, s); }
    cudaError_t e;
    if constexpr (Tiled) e = launch_tiled(k, grid, block, smem, s, args...);
    else e = launch(k, grid, block, smem, s, args...);
    if (eng->profiling) { b = next_event(eng); cudaEventRecord(b, s); eng->prof.push_back({name, a, b}); }
    eng->launch_counter++;
    return e;
}

// A zeroed device buffer.  The zeroing has finished when this returns: the
// engine stream is non-blocking, so a later cudaMemcpy on the default stream
// (the tables uploaded at creation) is not ordered after work queued on it.
int dalloc(gf_engine* eng, void** p, size_t bytes) {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        eng->err = "cudaMalloc(" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e);
        return GF_ENOMEM;
    }
    eng->allocs.push_back(*p);
    eng->bytes += bytes;
    e = cudaMemsetAsync(*p, 0, bytes, eng->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(eng->stream);
    if (e != cudaSuccess) { eng->err = std::string("cudaMemset: ") + cudaGetErrorString(e); return GF_ECUDA; }
    return GF_OK;
}

template <class T>
int dalloc_n(gf_engine* eng, T** p, size_t count) {
    return dalloc(eng, reinterpret_cast<void**>(p), count * sizeof(T));
}

// a real-valued device buffer of `count` elements of the run's precision
int dalloc_r(gf_engine* eng, double** p, size_t count) {
    return dalloc(eng, reinterpret_cast<void**>(p), count * eng->esz);
}

int alloc_field(gf_engine* eng, Field3& f, long l0, long l1, long l2) {
    f.on = true;
    f.len[0] = l0; f.len[1] = l1; f.len[2] = l2;
    for (int c = 0; c < 3; c++) {
        GF_TRY(dalloc_r(eng, &f.X[c], f.len[c]));
        GF_TRY(dalloc_r(eng, &f.A[c], f.len[c]));
        GF_TRY(dalloc_r(eng, &f.S0[c], f.len[c]));
        GF_TRY(dalloc_r(eng, &f.S1[c], f.len[c]));
        if (eng->mixed) GF_TRY(dalloc_r(eng, &f.C[c], f.len[c]));
    }
    return GF_OK;
}

// FP32 copy of a material table (member by member, same layout)
DevMatT<float> devmat_f32(const DevMat& d) {
    DevMatT<float> f;
    std::memset(&f, 0, sizeof(f));
    f.flags = d.flags; f.aniso = d.aniso; f.cubic_c = d.cubic_c;
    const double* src = &d.Ms;
    float* dst = &f.Ms;
    for (int q = 0; q < kDevMatReals; q++) dst[q] = (float)src[q];
    return f;
}

DevMat make_devmat(const Material& m, double dt) {
    DevMat d;
    std::memset(&d, 0, sizeof(d));
    d.flags = (m.fm ? MF_FM : 0u) | (m.afm ? MF_AFM : 0u) | (m.fe ? MF_FE : 0u) | (m.pec ? MF_PEC : 0u);
    d.aniso = (int)m.aniso_type;
    // magnetic_solver.cpp:84-87, 164-185, 206-208
    d.Ms = m.Ms;
    if (m.fm) {
        const double mu0 = kMu0;
        d.K1c = m.K1 / mu0 / m.Ms; d.K2c = m.K2 / mu0 / m.Ms;
        d.B1c = m.B1 / mu0 / m.Ms; d.B2c = m.B2 / mu0 / m.Ms;
        d.Aex = m.Aex;
        d.dA = m.iDMI / 2. / m.Aex;
        d.ex_coef = 2. / mu0 / m.Ms;
        d.dmi_coef = 2. * m.iDMI / mu0 / m.Ms;
        d.alpha = m.alpha;
        d.precess = -m.gyro / (1 + m.alpha * m.alpha) * dt;
        d.alpha_precess = m.alpha * d.precess;
    }
    d.Ms1 = m.Ms1; d.Ms2 = m.Ms2;
    if (m.afm) {
        // magnetic_AFM_solver.cpp:106-112, 181-191 (per sublattice)
        const double mu0 = kMu0;
        const double Ms[2] = {m.Ms1, m.Ms2}, K1[2] = {m.K1_1, m.K1_2}, B1[2] = {m.B1_1, m.B1_2}, B2[2] = {m.B2_1, m.B2_2};
        const double Aex[2] = {m.Aex1, m.Aex2}, gyro[2] = {m.gyro1, m.gyro2}, alpha[2] = {m.alpha1, m.alpha2};
        for (int s = 0; s < 2; s++) {
            d.aAex[s] = Aex[s];
            d.aK1c[s] = K1[s] / mu0 / Ms[s];
            d.aB1c[s] = B1[s] / mu0 / Ms[s]; d.aB2c[s] = B2[s] / mu0 / Ms[s];
            d.aJ[s] = -1. * m.J_AFM / mu0 / Ms[s];
            d.aex[s] = 2. / mu0 / Ms[s];
            d.aprec[s] = -gyro[s] / (1. + alpha[s] * alpha[s]) * dt;
            d.aaprec[s] = alpha[s] * d.aprec[s];
        }
        for (int a = 0; a < 3; a++) d.au[a] = m.uaxis[a];
    }
    // elastic
    bool cubic = true;
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) {
            d.cij[a][b] = m.cij[a][b];
            const bool in_pattern = (a < 3 && b < 3) || (a == b);
            if (!in_pattern && m.cij[a][b] != 0.) cubic = false;
        }
    d.cubic_c = cubic ? 1 : 0;
    d.dens_dt = dt / m.density;
    d.mass_damp = -dt * m.mass_damping;
    d.stiff_damp = m.stiff_damping / m.density;
    d.l100_15 = 1.5 * m.lam100; d.l111_15 = 1.5 * m.lam111;
    d.l100a1_075 = 0.5 * 1.5 * m.lam100_1; d.l100a2_075 = 0.5 * 1.5 * m.lam100_2;
    d.l111a1_075 = 0.5 * 1.5 * m.lam111_1; d.l111a2_075 = 0.5 * 1.5 * m.lam111_2;
    d.Q11 = m.Q11; d.Q12 = m.Q12; d.Q44 = m.Q44;
    // ferroelectric (ferroelectric_solver.cpp:704-717)
    d.a1 = m.a1; d.a11 = m.a11; d.a12 = m.a12; d.a111 = m.a111; d.a112 = m.a112; d.a123 = m.a123;
    d.a1111 = m.a1111; d.a1112 = m.a1112; d.a1122 = m.a1122; d.a1123 = m.a1123;
    d.tv1 = m.tv[0]; d.tv2 = m.tv[1]; d.tv3 = m.tv[2]; d.G11 = m.G11;
    if (m.fe) {
        d.fe_coef = -1. * dt / m.fe_mass;
        d.fe_damp = d.fe_coef * m.fe_damping;
    }
    d.tv4 = m.tv[3]; d.tv5 = m.tv[4]; d.tv6 = m.tv[5]; d.tv7 = m.tv[6]; d.tv8 = m.tv[7];
    d.f11 = m.f11; d.f12 = m.f12; d.f44x2 = 2. * m.f44;
    d.F11 = m.F11; d.F12 = m.F12; d.F44h = m.F44 / 2.;
    d.er = m.er; d.cond = m.cond;
    for (int k = 0; k < 3; k++) { d.comp[k] = m.comp[k]; d.wp[k] = m.wp[k]; d.rtau[k] = 1. / m.tau[k]; }
    return d;
}

// ---------------------------------------------------------------------------
// validation: what this engine implements
// ---------------------------------------------------------------------------
std::string unsupported(const Deck& d) {
    // kernels index cells and Yee vertices with 32-bit integers
    if ((double)(d.nx + 1) * (d.ny + 1) * (d.nz + 1) >= 2147483647.)
        return "grids with 2^31 or more Yee vertices are not supported (32-bit indexing)";
    if (d.elastostatic_1D || d.elastostatic_film || d.read_strain_ext)
        return "the 1-D and film elastostatic models and external strain (if_elastostatic_1D, if_elastostatic_film, if_read_strain_ext) are not supported by this engine";
    if (d.flexo && (d.elastostatic || d.in_straint0))
        return "flexoelectricity with a static strain (if_elastostatic or strain_stat.in) is not supported by this engine";
    if (d.num_materials > (unsigned)kMaxMat) return "more than 32 materials";
    for (size_t i = 0; i < d.mats.size(); i++) {
        const Material& m = d.mats[i];
        if (m.fm && m.aniso_type > 2) return "anisotropy_type must be 0, 1 or 2";
        if (m.fm && (m.Ms == 0. || m.Aex == 0.)) return "ferromagnetic material needs nonzero Ms and Aex";
        if (m.afm && (m.Ms1 == 0. || m.Ms2 == 0. || m.Aex1 == 0. || m.Aex2 == 0.))
            return "antiferromagnetic material needs nonzero Ms_AFM1/2 and Aex_AFM1/2";
        if (m.fm && m.afm) return "a material cannot be both ferromagnetic and antiferromagnetic";
        if (m.fe && m.fe_mass == 0.) return "ferroelectric material needs nonzero FE_mass";
        if (d.em_dynamic) {
            if (!(m.comp[0] == m.comp[0])) return "Drude weights sum to zero: the reference's normalisation yields NaN fields for this deck";
            // get_dJp_RK* runs for every material cell and divides by tao_e
            for (int k = 0; k < 3; k++)
                if (m.tau[k] == 0.) return "tao_e = 0: the reference's Drude update divides by it and its fields become NaN";
        }
    }
    if (d.elastodynamics) {
        if (d.nz < 5 && !d.abc_1D) return "the Liao boundary needs nz >= 5";
        if (d.nz < 2 && d.abc_1D) return "the elastic Mur boundary needs nz >= 2";
        if (d.strain_pulse && d.strain_z >= (unsigned)d.nz) return "input_strain_sourcez outside the grid";
        // the +z neighbour of get_dv_RK* is read out of the column when the
        // top face is not stress-free and nz-1 != ny-1 (elastic_dynamic_solver.cpp:1247)
        const long nx = d.nx, ny = d.ny, nz = d.nz;
        auto mc = [&](long i, long j, long k) { return d.material_cell[(size_t)((i * ny + j) * nz + k)]; };
        if (nz - 1 != ny - 1 && d.per_z) {
            for (long i = 0; i < nx; i++)
                for (long j = 0; j < ny; j++)
                    if (mc(i, j, 0) && mc(i, j, nz - 1)) return "periodic z with nz != ny and a solid top/bottom pair: the reference reads outside the array";
        }
        if (ny - 1 < nz - 1) {
            const long kq = ny - 1;
            for (long i = 0; i < nx; i++)
                for (long j = 0; j < ny; j++)
                    if (mc(i, j, kq) && mc(i, j, kq + 1) && !mc(i, j, 0))
                        return "reference quirk at k = ny-1 reads a vacuum cell's material";
        }
    }
    if (d.em_dynamic && d.planeEM) {
        if (d.nz_layer.empty()) return "plane-wave source needs at least one layer";
        if ((long)(d.nz_layer[0] / 5) > d.nz) return "plane-wave source plane outside the grid";
    }
    if (d.jf_input && d.em_dynamic) {
        if (d.jf_i1 >= (unsigned long)d.nx || d.jf_j1 >= (unsigned long)d.ny || d.jf_k1 >= (unsigned long)d.nz ||
            d.jf_i0 > d.jf_i1 || d.jf_j0 > d.jf_j1 || d.jf_k0 > d.jf_k1)
            return "J_f box outside the grid";
        if (d.jf_type > 6) return "Jf_input_type must be 0..6";
    }
    return "";
}

// physics the mixed form does not cover (none at present: every stage
// kernel has an FP32 instantiation)
std::string unsupported_mixed(const Deck&, const Params&) { return ""; }

void build_params(gf_engine* eng) {
    const Deck& d = eng->deck;
    Params& P = eng->P;
    std::memset(&P, 0, sizeof(P));
    P.nx = (int)d.nx; P.ny = (int)d.ny; P.nz = (int)d.nz; P.n = d.n();
    P.per_x = d.per_x; P.per_y = d.per_y; P.per_z = d.per_z;
    P.dx = d.dx; P.dy = d.dy; P.dz = d.dz; P.dt = d.dt;
    P.rdx = 1. / d.dx; P.rdy = 1. / d.dy; P.rdz = 1. / d.dz; P.rdt = 1. / d.dt;
    P.dt_e0 = d.dt / kE0; P.mdt_mu0 = -d.dt / kMu0;
    P.rot = d.orient_rotate;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) { P.Tg2c[i][j] = d.Tg2c[i][j]; P.Tc2g[i][j] = d.Tc2g[i][j]; }
    P.f.rdx = (float)P.rdx; P.f.rdy = (float)P.rdy; P.f.rdz = (float)P.rdz; P.f.rdt = (float)P.rdt;
    P.f.dt = (float)P.dt; P.f.dt_e0 = (float)P.dt_e0; P.f.mdt_mu0 = (float)P.mdt_mu0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) { P.f.Tg2c[i][j] = (float)P.Tg2c[i][j]; P.f.Tc2g[i][j] = (float)P.Tc2g[i][j]; }
    P.fm = d.any_fm; P.afm = d.any_afm; P.fe = d.any_fe; P.elastic = d.elastodynamics; P.em = d.em_dynamic;
    P.fe_mask = 0u; P.fm_mask = 0u;
    P.spin = (d.spin_pumping && (d.any_fm || d.any_afm)) ? 1 : 0;
    for (size_t q = 0; q < d.mats.size() && q < 32; q++) {
        if (d.mats[q].fe) P.fe_mask |= 1u << q;
        if (d.mats[q].fm) P.fm_mask |= 1u << q;
    }
    {
        long lo[3] = {d.nx, d.ny, d.nz}, hi[3] = {-1, -1, -1};
        for (long i = 0; i < d.nx; i++)
            for (long j = 0; j < d.ny; j++)
                for (long k = 0; k < d.nz; k++) {
                    const uint8_t id = d.material_cell[(size_t)((i * d.ny + j) * d.nz + k)];
                    if (!id || !d.mats[id - 1].fm) continue;
                    const long x[3] = {i, j, k};
                    for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], x[a]); hi[a] = std::max(hi[a], x[a]); }
                }
        if (hi[0] < 0) { lo[0] = lo[1] = lo[2] = 0; hi[0] = hi[1] = hi[2] = -1; }
        P.fm_i0 = lo[0]; P.fm_j0 = lo[1]; P.fm_k0 = lo[2];
        P.fm_bi = hi[0] - lo[0] + 1; P.fm_bj = hi[1] - lo[1] + 1; P.fm_bk = hi[2] - lo[2] + 1;
    }
    {
        long lo[3] = {d.nx, d.ny, d.nz}, hi[3] = {-1, -1, -1};
        for (long i = 0; i < d.nx; i++)
            for (long j = 0; j < d.ny; j++)
                for (long k = 0; k < d.nz; k++) {
                    const uint8_t id = d.material_cell[(size_t)((i * d.ny + j) * d.nz + k)];
                    if (!id || !d.mats[id - 1].afm) continue;
                    const long x[3] = {i, j, k};
                    for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], x[a]); hi[a] = std::max(hi[a], x[a]); }
                }
        if (hi[0] < 0) { lo[0] = lo[1] = lo[2] = 0; hi[0] = hi[1] = hi[2] = -1; }
        P.afm_i0 = lo[0]; P.afm_j0 = lo[1]; P.afm_k0 = lo[2];
        P.afm_bi = hi[0] - lo[0] + 1; P.afm_bj = hi[1] - lo[1] + 1; P.afm_bk = hi[2] - lo[2] + 1;
    }
    P.elasto_on = d.elasto_on; P.elasto_back = d.elasto_back && d.elastodynamics;
    P.em_fromM = d.em_fromM && d.em_dynamic && (d.any_fm || d.any_afm);
    P.em_fromP = d.em_fromP && d.em_dynamic && d.any_fe;
    P.em_back_M = d.em_back_M && d.em_dynamic;
    P.em_back_P = d.em_back_P && d.em_dynamic;
    P.has_hext_nonunif = d.read_Hext_nonunif;
    P.abc_1D = d.abc_1D; P.abc_elast_onlytop = d.abc_elast_onlytop; P.abc_em_onlytop = d.abc_em_onlytop;
    P.prescribed_m = (d.prescribed_m && d.any_fm) ? 1 : 0;
    P.pec_xy = d.pec_xy; P.pec_z = d.pec_z; P.mag_1D = d.mag_1D;
    P.mag1d_em = (d.mag_1D && d.em_dynamic && d.em_fromM) ? 1 : 0;
    // the elastic boundary planes inside the RK update: the Liao history
    // needs planes 1-4, and a displacement source on a boundary plane
    // would be overwritten in the other order
    P.el_bc_fused = (d.elastodynamics && d.nz >= 5 &&
                     !(d.strain_pulse && (d.strain_z == 0 || (long)d.strain_z + 1 >= (long)d.nz))) ? 1 : 0;
    P.flexo = (d.flexo && d.any_fe) ? 1 : 0;
    P.elastostatic = d.elastostatic ? 1 : 0;
    P.drude = 0; P.pec = 0;
    if (d.em_dynamic)
        for (const Material& m : d.mats) {
            for (int k = 0; k < 3; k++) if (m.wp[k] != 0.) P.drude = 1;
            if (m.pec) P.pec = 1;
        }
    P.liao_w = d.liao_w;

    // sound speeds of the first and last z planes (elastic_initialize.cpp:43-80)
    auto first_mat = [&](long k) -> const Material* {
        for (long i = 0; i < d.nx; i++)
            for (long j = 0; j < d.ny; j++) {
                uint8_t id = d.material_cell[(size_t)((i * d.ny + j) * d.nz + k)];
                if (id) return &d.mats[id - 1];
            }
        return nullptr;
    };
    double c11_1 = 0., c44_1 = 0., rho_1 = 1.e-8, c11_l = 0., c44_l = 0., rho_l = 1.e-8;
    if (const Material* m = first_mat(0)) { c11_1 = m->c11; c44_1 = m->c44; rho_1 = m->density; }
    if (const Material* m = first_mat(d.nz - 1)) { c11_l = m->c11; c44_l = m->c44; rho_l = m->density; }
    P.vs_long_1st = std::sqrt((c11_1 / rho_1)); P.vs_tran_1st = std::sqrt((c44_1 / rho_1));
    P.vs_long_last = std::sqrt((c11_l / rho_l)); P.vs_tran_last = std::sqrt((c44_l / rho_l));
    const double dz = d.dz, dt = d.dt;
    const double vs[4] = {P.vs_long_1st, P.vs_tran_1st, P.vs_long_last, P.vs_tran_last};
    for (int a = 0; a < 4; a++) {
        P.mur_el_half[a] = (2. * dz - vs[a] * dt) / (2. * dz + vs[a] * dt);
        P.mur_el_full[a] = (dz - vs[a] * dt) / (dz + vs[a] * dt);
    }
    P.source_z = d.strain_z;
    P.strain_pulse = d.strain_pulse; P.strain_type = (int)d.strain_type;
    P.strain_comp = d.strain_comp == 'y' ? 1 : (d.strain_comp == 'z' ? 2 : 0);

    // Maxwell Mur coefficients (EMdynamic_initialize.cpp:24-56)
    auto first_er = [&](long k) -> double {
        for (long i = 0; i < d.nx; i++)
            for (long j = 0; j < d.ny; j++) {
                uint8_t id = d.material_cell[(size_t)((i * d.ny + j) * d.nz + k)];
                if (id) return std::sqrt(d.mats[id - 1].er);
            }
        return 1.;
    };
    const double sq_bot = first_er(0), sq_top = first_er(d.nz - 1);
    const double c = kC0, dx = d.dx, dy = d.dy;
    P.c_top_half = (2. * dz - c / sq_top * dt) / (2. * dz + c / sq_top * dt);
    P.c_bot_half = (2. * dz - c / sq_bot * dt) / (2. * dz + c / sq_bot * dt);
    P.c_x_half = (2. * dx - c * dt) / (2. * dx + c * dt);
    P.c_y_half = (2. * dy - c * dt) / (2. * dy + c * dt);
    P.c_top = (dz - c / sq_top * dt) / (dz + c / sq_top * dt);
    P.c_bot = (dz - c / sq_bot * dt) / (dz + c / sq_bot * dt);
    P.c_x = (dx - c * dt) / (dx + c * dt);
    P.c_y = (dy - c * dt) / (dy + c * dt);
    P.plane_z = d.nz_layer.empty() ? 0 : (long)(d.nz_layer[0] / 5);
    P.planeEM = d.planeEM && d.em_dynamic;
    P.jf_on = d.jf_input && d.em_dynamic;
    P.jf_type = (int)d.jf_type;
    P.jf_comp = d.jf_comp == 'y' ? 1 : (d.jf_comp == 'z' ? 2 : 0);
    P.jf_i0 = (long)d.jf_i0; P.jf_i1 = (long)d.jf_i1; P.jf_j0 = (long)d.jf_j0; P.jf_j1 = (long)d.jf_j1;
    P.jf_k0 = (long)d.jf_k0; P.jf_k1 = (long)d.jf_k1;
}

// ---------------------------------------------------------------------------
// time-dependent drive of one step (host, reference expressions)
// ---------------------------------------------------------------------------
void step_drive(gf_engine* eng, StepDrive& sd) {
    const Deck& d = eng->deck;
    const double PI = kPi;
    const double dt = d.dt;
    // time_marching_device_serial (global.cpp:512-549)
    eng->t_host = eng->t_host + dt;
    const double t = eng->t_host;
    sd.t = t;
    if (d.prescribe_E) {
        if (eng->presc_E < d.n_prescribe_E && (t - dt) > d.tE[eng->presc_E]) eng->presc_E = eng->presc_E + 1;
        if (eng->presc_E < d.n_prescribe_E) { eng->Eext_cur[0] = d.Ex[eng->presc_E]; eng->Eext_cur[1] = d.Ey[eng->presc_E]; eng->Eext_cur[2] = d.Ez[eng->presc_E]; }
        else { eng->Eext_cur[0] = eng->Eext_cur[1] = eng->Eext_cur[2] = 0.; }
    }
    if (d.prescribe_H) {
        if (eng->presc_H < d.n_prescribe_H && (t - dt) > d.tH[eng->presc_H]) eng->presc_H = eng->presc_H + 1;
        if (eng->presc_H < d.n_prescribe_H) { eng->Hext_cur[0] = d.Hx[eng->presc_H]; eng->Hext_cur[1] = d.Hy[eng->presc_H]; eng->Hext_cur[2] = d.Hz[eng->presc_H]; }
        else { eng->Hext_cur[0] = eng->Hext_cur[1] = eng->Hext_cur[2] = 0.; }
    }
    // local times of the four stages
    const double lt_ext[4] = {t - dt, t - dt * 0.5, t - dt * 0.5, t};
    // prescribed m of the k = 0 ferromagnetic cells after each update
    // (update_prescribed_m_half / _full / update_prescribed_m,
    // magnetic_solver.cpp:1891-1960): at t - dt/2 after stages 1-2, at t
    // after stage 3 and the step
    double pm[4][3] = {};
    if (d.prescribed_m) {
        const double m0 = std::sin(d.precess_angle / 180. * PI);
        const double omega = 2. * PI * d.precess_freq;
        for (int s = 0; s < 4; s++) {
            const double tt = (s < 2) ? t - dt * 0.5 : t;
            pm[s][0] = std::sqrt((1. - m0 * m0));
            pm[s][1] = m0 * std::sin(omega * tt);
            pm[s][2] = m0 * std::cos(omega * tt);
        }
    }
    // static + alternating H of each stage (update_external_Hfield*, magnetic_solver.cpp:1834-1861)
    double Hf[4][3];
    for (int s = 0; s < 4; s++)
        for (int a = 0; a < 3; a++) Hf[s][a] = d.Hext_stat[a] + d.Hext_altr[a] * std::sin(2. * PI * d.H_altr_freq[a] * lt_ext[s]);
    for (int s = 0; s < 4; s++) {
        StageDrive& st = sd.st[s];
        std::memset(&st, 0, sizeof(st));
        for (int a = 0; a < 3; a++) st.pm[a] = pm[s][a];
        for (int a = 0; a < 3; a++) {
            // With a prescribed table the ferromagnet keeps the shared Hext
            // (magnetic_solver.cpp:35-40) while get_dm_AFM_RK* always
            // recomputes it (magnetic_AFM_solver.cpp:63, 491, 919, 1347), so
            // the ferromagnet's stages 2-4 see the value the antiferromagnet
            // set one stage earlier.
            st.Hext_afm[a] = Hf[s][a];
            if (!d.prescribe_H) st.Hext[a] = Hf[s][a];
            else if (d.any_afm && s > 0) st.Hext[a] = Hf[s - 1][a];
            else st.Hext[a] = eng->Hext_cur[a];
            st.Eext[a] = d.prescribe_E ? eng->Eext_cur[a]
                                       : d.Eext_stat[a] + d.Eext_altr[a] * std::sin(2. * PI * d.E_altr_freq[a] * lt_ext[s]);
        }
        // surface traction (type 3), get_dv_RK*
        {
            double tv;
            if (s == 0) tv = t - dt - 5.0 * d.sigma_gauss;
            else if (s < 3) tv = t - 0.5 * dt - 5.0 * d.sigma_gauss;
            else tv = t - 5.0 * d.sigma_gauss;
            st.traction = d.amp_gauss * std::exp(-1. * std::pow(tv, 2.) / (2. * std::pow(d.sigma_gauss, 2.)));
        }
        // displacement source written after the stage update
        // (update_Du_Gaussian_half for stages 1-2, _full for 3, final for 4)
        {
            const double vs = (d.strain_comp == 'z') ? eng->P.vs_long_1st : eng->P.vs_tran_1st;
            const bool half = (s < 2);
            const double tl = half ? (t - 0.5 * dt) : t;
            st.usrc_on = 0;
            if (d.strain_type == 1 && t < 12.5 * d.sigma_gauss) {
                st.usrc_on = 1;
                st.usrc = d.amp_gauss * 1.6487210 * d.sigma_gauss * vs *
                          std::exp(-1. * std::pow((tl - 5.0 * d.sigma_gauss), 2.) / (2. * d.sigma_gauss * d.sigma_gauss));
            } else if (d.strain_type == 2) {
                st.usrc_on = 1;
                const double val = d.amp_gauss * vs / 2. / PI / d.sigma_gauss * (std::cos(2. * PI * d.sigma_gauss * (tl)) - 1);
                if (d.strain_cycles == 0) st.usrc = val;
                else st.usrc = (tl <= static_cast<double>(d.strain_cycles) / d.sigma_gauss) ? val : 0.;
            }
        }
        // free-current source value (update_Jf_input / _half / _full)
        if (d.jf_input) {
            // stage 3 keeps the stage-2 value (get_dE_RK3 does not refresh J_f)
            const int v = (s == 0) ? 0 : (s < 3 ? 1 : 2);
            const double tl = (v == 0) ? (t - dt) : (v == 1 ? (t - 0.5 * dt) : t);
            double val = 0.;
            if (d.jf_type < 3) {
                double temporal;
                if (v == 0) temporal = std::sin(2. * PI * d.jf_freq * (t - dt));
                else if (v == 1) temporal = std::sin(2. * PI * d.jf_freq * (t - 0.5 * dt));
                else temporal = std::sin(2. * PI * d.jf_freq * t);
                val = d.jf_amp * temporal;
            } else if (d.jf_type == 3) {
                double temporal = 0.;
                if (tl <= static_cast<double>(d.jf_cycles) / d.jf_freq) {
                    if (v == 0) temporal = std::sin(2. * PI * d.jf_freq * (t - dt));
                    else if (v == 1) temporal = std::sin(2. * PI * d.jf_freq * (t - 0.5 * dt));
                    else temporal = std::sin(2. * PI * d.jf_freq * (t));
                }
                val = d.jf_amp * temporal;
            } else if (d.jf_type == 4 || d.jf_type == 5) {
                double tv;
                if (v == 0) tv = t - dt - 5. * d.jf_freq;
                else if (v == 1) tv = t - 0.5 * dt - 5. * d.jf_freq;
                else tv = t - 5. * d.jf_freq;
                if (d.jf_type == 4) val = d.jf_amp * std::exp(-1. * std::pow(tv, 2.) / (2. * std::pow(d.jf_freq, 2.)));
                else val = d.jf_amp * std::sqrt(std::exp(1.)) * tv / d.jf_freq * std::exp(-1. * std::pow(tv, 2.) / (2. * std::pow(d.jf_freq, 2.)));
            } else if (d.jf_type == 6) {
                double tv, sarg;
                if (v == 0) { tv = t - dt - 5. * d.jf_sigma; sarg = (t - dt); }
                else if (v == 1) { tv = t - 0.5 * dt - 5. * d.jf_sigma; sarg = (t - 0.5 * dt); }
                else { tv = t - 5. * d.jf_sigma; sarg = t; }
                if (v == 2) val = d.jf_amp * std::exp(-1. * std::pow(tv, 2.) / (2. * std::pow(d.jf_sigma, 2.))) * std::sin(2. * PI * d.jf_freq * t);
                else val = d.jf_amp * std::exp(-1. * std::pow(tv, 2.) / (2. * std::pow(d.jf_sigma, 2.))) * std::sin(2. * PI * d.jf_freq * sarg);
            }
            st.jf = val;
        }
        // plane wave (update_planeEM_half for stages 1-2, _full for 3 and the final update)
        for (int a = 0; a < 3; a++) {
            if (s < 2) st.plane[a] = d.planeEM_E[a] * std::sin(2. * PI * d.planeEM_freq[a] * (t - 0.5 * dt));
            else st.plane[a] = d.planeEM_E[a] * std::sin(2. * PI * d.planeEM_freq[a] * t);
        }
    }
}

// ---------------------------------------------------------------------------
// stage IO tables
// ---------------------------------------------------------------------------
F3 f3(double* const* p) { F3 r; for (int c = 0; c < 3; c++) r.c[c] = p[c]; return r; }

void set_io_field(const Field3& f, int parity, int s, F3& in, F3& x, F3& acc, F3& out) {
    // parity 0: X = f.X, A = f.A ; parity 1: roles swapped
    double* const* X = parity ? f.A : f.X;
    double* const* A = parity ? f.X : f.A;
    x = f3(X);
    acc = f3(A);
    if (s == 0) { in = f3(X); out = f3(f.S0); }
    else if (s == 1) { in = f3(f.S0); out = f3(f.S1); }
    else if (s == 2) { in = f3(f.S1); out = f3(f.S0); }
    else { in = f3(f.S0); out = f3(A); }
}

void build_io(gf_engine* eng) {
    for (int par = 0; par < 2; par++)
        for (int s = 0; s < 4; s++) {
            StageIO& io = eng->io[par][s];
            std::memset(&io, 0, sizeof(io));
            if (eng->m.on) set_io_field(eng->m, par, s, io.m_in, io.m_x, io.m_acc, io.m_out);
            if (eng->a1.on) set_io_field(eng->a1, par, s, io.a1_in, io.a1_x, io.a1_acc, io.a1_out);
            if (eng->a2.on) set_io_field(eng->a2, par, s, io.a2_in, io.a2_x, io.a2_acc, io.a2_out);
            if (eng->p.on) set_io_field(eng->p, par, s, io.p_in, io.p_x, io.p_acc, io.p_out);
            if (eng->q.on) set_io_field(eng->q, par, s, io.q_in, io.q_x, io.q_acc, io.q_out);
            if (eng->u.on) set_io_field(eng->u, par, s, io.u_in, io.u_x, io.u_acc, io.u_out);
            if (eng->v.on) set_io_field(eng->v, par, s, io.v_in, io.v_x, io.v_acc, io.v_out);
            if (eng->E.on) set_io_field(eng->E, par, s, io.E_in, io.E_x, io.E_acc, io.E_out);
            if (eng->H.on) set_io_field(eng->H, par, s, io.H_in, io.H_x, io.H_acc, io.H_out);
            for (int pole = 0; pole < 3; pole++)
                if (eng->jp[pole].on)
                    set_io_field(eng->jp[pole], par, s, io.jp_in[pole], io.jp_x[pole], io.jp_acc[pole], io.jp_out[pole]);
            io.dm = f3(eng->dm);
            io.da1 = f3(eng->da1);
            io.da2 = f3(eng->da2);
            io.force_store = f3(eng->force_store);
            io.force = f3(eng->force);
            io.Hstat = f3(eng->Hstat);
            io.Estat = f3(eng->Estat);
            io.Hnu = f3(eng->Hnu);
            for (int a = 0; a < 9; a++) io.fg[a] = eng->fg[a];
            for (int a = 0; a < 6; a++) io.strain_c[a] = eng->strain_c[a];
            for (int a = 0; a < 6; a++) { io.sg[a] = eng->flexo_sg[a]; io.pge[a] = eng->flexo_pge[a]; }
            for (int a = 0; a < 6; a++) { io.eps0_c[a] = eng->es_eps[a]; io.eig0_c[a] = eng->es_eig[a]; }
            io.liao_hist = eng->liao_hist;
            io.liao_last = eng->liao_last;
            io.msrc = eng->demag_src_fused ? eng->Mfft : nullptr;
            io.mid = eng->mid;
            io.mats = eng->mats;
            io.drive = eng->drive;
            io.drive_mask = (unsigned long long)(kDriveCap - 1);
            io.step = eng->step_ctr;
            io.jf_kfac = eng->jf_kfac;
            io.ishe_coef = eng->ishe_coef;
            io.ishe_src = eng->ishe_src;
            for (int c = 0; c < 3; c++) io.ecls[c] = eng->ecls[c];
        }
}

// float views of the run's buffers (mixed form)
F3T<float> f3f(double* const* p) {
    F3T<float> r;
    for (int c = 0; c < 3; c++) r.c[c] = reinterpret_cast<float*>(p[c]);
    return r;
}
void set_io_field_f(const Field3& f, int parity, int s, F3T<float>& in, F3T<float>& x, F3T<float>& acc,
                    F3T<float>& out, F3T<float>& cmp) {
    double* const* X = parity ? f.A : f.X;
    double* const* A = parity ? f.X : f.A;
    x = f3f(X);
    acc = f3f(A);
    cmp = f3f(f.C);
    if (s == 0) { in = f3f(X); out = f3f(f.S0); }
    else if (s == 1) { in = f3f(f.S0); out = f3f(f.S1); }
    else if (s == 2) { in = f3f(f.S1); out = f3f(f.S0); }
    else { in = f3f(f.S0); out = f3f(A); }
}

void build_io_mixed(gf_engine* eng) {
    for (int par = 0; par < 2; par++)
        for (int s = 0; s < 4; s++) {
            StageIOT<float>& io = eng->iof[par][s];
            std::memset(&io, 0, sizeof(io));
            if (eng->m.on) set_io_field_f(eng->m, par, s, io.m_in, io.m_x, io.m_acc, io.m_out, io.m_cmp);
            if (eng->a1.on) set_io_field_f(eng->a1, par, s, io.a1_in, io.a1_x, io.a1_acc, io.a1_out, io.a1_cmp);
            if (eng->a2.on) set_io_field_f(eng->a2, par, s, io.a2_in, io.a2_x, io.a2_acc, io.a2_out, io.a2_cmp);
            for (int pole = 0; pole < 3; pole++)
                if (eng->jp[pole].on)
                    set_io_field_f(eng->jp[pole], par, s, io.jp_in[pole], io.jp_x[pole], io.jp_acc[pole], io.jp_out[pole],
                                   io.jp_cmp[pole]);
            if (eng->p.on) set_io_field_f(eng->p, par, s, io.p_in, io.p_x, io.p_acc, io.p_out, io.p_cmp);
            if (eng->q.on) set_io_field_f(eng->q, par, s, io.q_in, io.q_x, io.q_acc, io.q_out, io.q_cmp);
            if (eng->u.on) set_io_field_f(eng->u, par, s, io.u_in, io.u_x, io.u_acc, io.u_out, io.u_cmp);
            if (eng->v.on) set_io_field_f(eng->v, par, s, io.v_in, io.v_x, io.v_acc, io.v_out, io.v_cmp);
            if (eng->E.on) set_io_field_f(eng->E, par, s, io.E_in, io.E_x, io.E_acc, io.E_out, io.E_cmp);
            if (eng->H.on) set_io_field_f(eng->H, par, s, io.H_in, io.H_x, io.H_acc, io.H_out, io.H_cmp);
            io.dm = f3f(eng->dm);
            io.da1 = f3f(eng->da1);
            io.da2 = f3f(eng->da2);
            io.force_store = f3f(eng->force_store);
            io.force = f3f(eng->force);
            io.Hstat = f3f(eng->Hstat);
            io.Estat = f3f(eng->Estat);
            io.Hnu = f3f(eng->Hnu);
            for (int a = 0; a < 9; a++) io.fg[a] = reinterpret_cast<float*>(eng->fg[a]);
            for (int a = 0; a < 6; a++) io.strain_c[a] = reinterpret_cast<float*>(eng->strain_c[a]);
            for (int a = 0; a < 6; a++) {
                io.sg[a] = reinterpret_cast<float*>(eng->flexo_sg[a]);
                io.pge[a] = reinterpret_cast<float*>(eng->flexo_pge[a]);
                io.eps0_c[a] = reinterpret_cast<const float*>(eng->es_eps[a]);
                io.eig0_c[a] = reinterpret_cast<const float*>(eng->es_eig[a]);
            }
            io.liao_hist = reinterpret_cast<float*>(eng->liao_hist);
            io.liao_last = reinterpret_cast<float*>(eng->liao_last);
            io.msrc = eng->demag_src_fused ? reinterpret_cast<float*>(eng->Mfft) : nullptr;
            io.mid = eng->mid;
            io.mats = eng->mats_f;
            io.drive = eng->drive;
            io.drive_mask = (unsigned long long)(kDriveCap - 1);
            io.step = eng->step_ctr;
            io.jf_kfac = reinterpret_cast<const float*>(eng->jf_kfac);
            io.ishe_coef = reinterpret_cast<const float*>(eng->ishe_coef);
            io.ishe_src = eng->ishe_src;
            for (int c = 0; c < 3; c++) io.ecls[c] = eng->ecls[c];
        }
}

// ---------------------------------------------------------------------------
// one RK4 step: kernel sequence in the reference's data order
// ---------------------------------------------------------------------------
// Shared-memory opt-in and the x-chunk of the tiled elastic kernel.  A
// block of `L` planes costs L+2 plane passes (one halo plane each side), so
// the chunk count minimises waves x (L+2) over the blocks that fit at once.
template <class R>
int set_elastic_smem(gf_engine* eng, int smem) {
    GF_CU(cudaFuncSetAttribute(k_elastic_tile<0, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    GF_CU(cudaFuncSetAttribute(k_elastic_tile<1, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    GF_CU(cudaFuncSetAttribute(k_elastic_tile<2, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    GF_CU(cudaFuncSetAttribute(k_elastic_tile<3, true, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    GF_CU(cudaFuncSetAttribute(k_elastic_tile<0, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    GF_CU(cudaFuncSetAttribute(k_elastic_tile<1, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    GF_CU(cudaFuncSetAttribute(k_elastic_tile<2, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    GF_CU(cudaFuncSetAttribute(k_elastic_tile<3, false, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return GF_OK;
}

#ifndef GF_MIXED_TU
int setup_elastic_tile(gf_engine* eng) {
    const Params& P = eng->P;
    eng->el_nmat = (int)eng->deck.mats.size();
    eng->el_smem = eng->mixed ? etile::smem_bytes<float>(eng->el_nmat) : etile::smem_bytes<double>(eng->el_nmat);
    const int smem = (int)eng->el_smem;
    eng->el_cubic = true;
    for (const Material& m : eng->deck.mats)
        for (int a = 0; a < 6; a++)
            for (int b = 0; b < 6; b++)
                if (!((a < 3 && b < 3) || a == b) && m.cij[a][b] != 0.) eng->el_cubic = false;
    int per_sm = 1, sms = 1;
    if (eng->mixed) {
        GF_TRY(gf_mixed_elastic_setup(eng, smem, &per_sm));
    } else {
        GF_TRY(set_elastic_smem<double>(eng, smem));
        GF_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_elastic_tile<1, false, double>, etile::NT, eng->el_smem));
    }
    GF_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, eng->device));
    if (per_sm < 1) { eng->err = "elastic tile does not fit on an SM"; return GF_ECUDA; }
    long slots = (long)per_sm * (sms > 0 ? sms : 1);
    // In the mixed form without magnets the TDGL and Maxwell kernels do not
    // wait for the tile and share the SMs with it: the tile's blocks are held
    // to three fifths of the resident slots, which leaves them room (128^3
    // ferroelectric FP32 step, ms, by planes per block and share of the
    // slots: 16 / 86 % 1.355, 19 / 76 % 1.338, 22 / 65 % 1.327, 26 / 54 %
    // 1.322, 32 / 43 % 1.351; the FP64 step, whose TDGL kernel waits for the
    // tile, measured slower with the smaller share, 2.379 -> 2.395 ms, and so
    // did the FP32 magnetoelastic film, whose LLG kernel waits for it, 0.878
    // -> 1.014 ms)
    if (eng->mixed && P.fe && !(P.fm || P.afm)) slots = std::max<long>(1, slots * 3 / 5);
    const long tiles = (long)((P.nz + etile::TK - 1) / etile::TK) * ((P.ny + etile::TJ - 1) / etile::TJ);
    long best_cost = -1;
    for (long c = 1; c <= P.nx; c++) {
        const long L = (P.nx + c - 1) / c;
        const long blocks = tiles * ((P.nx + L - 1) / L);
        const long cost = ((blocks + slots - 1) / slots) * (L + 2);
        if (best_cost < 0 || cost < best_cost) { best_cost = cost; eng->el_chunk = (int)L; }
    }
    return GF_OK;
}
#endif  // GF_MIXED_TU

template <class R> const StageIOT<R>& stage_io(const gf_engine* eng, int parity, int s);
template <class R> const LLGTablesT<R>* llg_tables(const gf_engine* eng);
#ifdef GF_MIXED_TU
template <> const StageIOT<float>& stage_io<float>(const gf_engine* eng, int parity, int s) { return eng->iof[parity][s]; }
template <> const LLGTablesT<float>* llg_tables<float>(const gf_engine* eng) { return eng->llg_tab_f; }
#else
template <> const StageIOT<double>& stage_io<double>(const gf_engine* eng, int parity, int s) { return eng->io[parity][s]; }
template <> const LLGTablesT<double>* llg_tables<double>(const gf_engine* eng) { return eng->llg_tab; }
#endif

// magnetostatic field of magnetisation m into Hstat (FFT, demag factors or
// the 1-D model), FP64 form
// src_ready: the stage's LLG kernel has already written the transform's
// input (StageIOT::msrc), so the source kernel is skipped
int demag_solve(gf_engine* eng, F3 m, F3 a1, F3 a2, bool counted, bool src_ready = false) {
    const Params& P = eng->P;
    cudaStream_t st = eng->stream;
    const unsigned bn = blocks_for(P.n, kThreads);
    auto L = [&](const char* name, auto k, dim3 g, dim3 b, auto... args) -> cudaError_t {
        return counted ? klaunch(eng, name, k, g, b, 0, st, args...) : launch(k, g, b, 0, st, args...);
    };
    if (eng->demag_mode == 0) {
        if (!src_ready)
            GF_CU(L("k_mag_source", k_mag_source, dim3(bn), dim3(kThreads), P, (const DevMat*)eng->mats, (const uint8_t*)eng->mid,
                    m, a1, a2, 0, eng->Mfft, f3(eng->Hstat), 0., 0., 0.));
        GF_FFT(cufftExecD2Z(eng->plan_r2c, eng->Mfft, eng->Mk));
        const long n21 = (long)P.nx * P.ny * (P.nz / 2 + 1);
        const double vol_neg = -P.dx * P.dy * P.dz;
        GF_CU(L("k_demag_mul", k_demag_mul, dim3(blocks_for(n21, kThreads)), dim3(kThreads), n21, vol_neg,
                (const cuDoubleComplex*)eng->Mk, (const cuDoubleComplex*)eng->Nk, (cuDoubleComplex*)eng->Mk));
        // the inverse transform lands in H_stat itself (H_stat is a view of
        // the FFT buffer in the FFT mode)
        GF_FFT(cufftExecZ2D(eng->plan_c2r, eng->Mk, eng->Mfft));
    } else {
        GF_CU(L("k_mag_source", k_mag_source, dim3(bn), dim3(kThreads), P, (const DevMat*)eng->mats, (const uint8_t*)eng->mid,
                m, a1, a2, eng->demag_mode, (double*)nullptr, f3(eng->Hstat), eng->deck.demag_fac[0], eng->deck.demag_fac[1],
                eng->deck.demag_fac[2]));
    }
    return GF_OK;
}

// the same in the mixed form: FP32 source, R2C, spectra product, C2R
int demag_solve_f32(gf_engine* eng, F3T<float> m, F3T<float> a1, F3T<float> a2, bool counted, bool src_ready = false) {
    const Params& P = eng->P;
    cudaStream_t st = eng->stream;
    const unsigned bn = blocks_for(P.n, kThreads);
    auto L = [&](const char* name, auto k, dim3 g, dim3 b, auto... args) -> cudaError_t {
        return counted ? klaunch(eng, name, k, g, b, 0, st, args...) : launch(k, g, b, 0, st, args...);
    };
    float* M3 = reinterpret_cast<float*>(eng->Mfft);
    cufftComplex* Mk = reinterpret_cast<cufftComplex*>(eng->Mk);
    if (eng->demag_mode == 0) {
        if (!src_ready)
            GF_CU(L("k_mag_source", k_mag_source_f32, dim3(bn), dim3(kThreads), P, (const DevMatT<float>*)eng->mats_f,
                    (const uint8_t*)eng->mid, m, a1, a2, 0, M3, f3f(eng->Hstat), 0.f, 0.f, 0.f));
        GF_FFT(cufftExecR2C(eng->plan_r2c, M3, Mk));
        const long n21 = (long)P.nx * P.ny * (P.nz / 2 + 1);
        const float inv_vol_neg = (float)(-1. / (P.dx * P.dy * P.dz));
        GF_CU(L("k_demag_mul", k_demag_mul_f32, dim3(blocks_for(n21, kThreads)), dim3(kThreads), n21, inv_vol_neg,
                (const cuComplex*)Mk, (const float*)eng->Nr, (cuComplex*)Mk));
        GF_FFT(cufftExecC2R(eng->plan_c2r, Mk, M3));     // into H_stat (a view of M3)
    } else {
        GF_CU(L("k_mag_source", k_mag_source_f32, dim3(bn), dim3(kThreads), P, (const DevMatT<float>*)eng->mats_f,
                (const uint8_t*)eng->mid, m, a1, a2, eng->demag_mode, (float*)nullptr, f3f(eng->Hstat), (float)eng->deck.demag_fac[0],
                (float)eng->deck.demag_fac[1], (float)eng->deck.demag_fac[2]));
    }
    return GF_OK;
}

constexpr int kElecBlocks = 592;

// `iters` fixed-point iterations of the electrostatic solve with the stage
// polarisation p, updating Hstat's electric counterpart Estat in place; with
// tol > 0 (set-up only) stop early once max|E_new - E_old| <= tol max|E_new|
int elec_solve(gf_engine* eng, F3 p, bool counted, int iters, double tol, int* used) {
    const Params& P = eng->P;
    cudaStream_t st = eng->stream;
    const unsigned bn = blocks_for(P.n, kThreads);
    const long n21 = (long)P.nx * P.ny * (P.nz / 2 + 1);
    auto L = [&](const char* name, auto k, dim3 g, dim3 b, auto... args) -> cudaError_t {
        return counted ? klaunch(eng, name, k, g, b, 0, st, args...) : launch(k, g, b, 0, st, args...);
    };
    const double inv = 1. / (kE0 * eng->elec_erh * (double)P.n);
    std::vector<double> bm(2 * kElecBlocks);
    int it = 0;
    for (; it < iters; it++) {
        GF_CU(L("k_elec_source", k_elec_source, dim3(bn), dim3(kThreads), P, (const DevMat*)eng->mats, (const uint8_t*)eng->mid,
                p, f3(eng->Estat), eng->elec_erh, eng->elec_q));
        GF_FFT(cufftExecD2Z(eng->elec_r2c, eng->elec_q, eng->elec_qk));
        GF_CU(L("k_elec_mul", k_elec_mul, dim3(blocks_for(n21, kThreads)), dim3(kThreads), P, n21, (const double*)eng->elec_k[0],
                (const double*)eng->elec_k[1], (const double*)eng->elec_k[2], inv, eng->elec_qk));
        GF_FFT(cufftExecZ2D(eng->elec_c2r, eng->elec_qk, eng->elec_q));
        GF_CU(L("k_elec_update", k_elec_update, dim3(kElecBlocks), dim3(256), P, (const double*)eng->elec_q, f3(eng->Estat),
                tol > 0. ? eng->elec_blockmax : (double*)nullptr));
        if (tol > 0.) {
            GF_CU(cudaMemcpyAsync(bm.data(), eng->elec_blockmax, sizeof(double) * bm.size(), cudaMemcpyDeviceToHost, st));
            GF_CU(cudaStreamSynchronize(st));
            double md = 0., me = 0.;
            for (int b = 0; b < kElecBlocks; b++) { md = std::max(md, bm[2 * b]); me = std::max(me, bm[2 * b + 1]); }
            if (md <= tol * me) { it++; break; }
        }
    }
    if (used) *used = it;
    return GF_OK;
}

// TDGL kernel of stage S on stream st
template <int S, class R>
int enqueue_fe(gf_engine* eng, const StageIOT<R>& io, cudaStream_t st) {
    const Params& P = eng->P;
    const dim3 g(blocks_for((long)P.ny * P.nz, kThreads), (unsigned)P.nx);
    if (P.flexo) GF_CU(klaunch(eng, "k_fe", k_fe<S, R, true>, g, dim3(kThreads), 0, st, P, io));
    else GF_CU(klaunch(eng, "k_fe", k_fe<S, R, false>, g, dim3(kThreads), 0, st, P, io));
    return GF_OK;
}

// Maxwell kernels of stage S on stream st: the Yee update, then the plane
// source, the Mur boundaries, PEC and the Drude currents, in that order
template <int S, class R>
int enqueue_em(gf_engine* eng, const StageIOT<R>& io, cudaStream_t st) {
    const Params& P = eng->P;
    const long nx = P.nx, ny = P.ny, nz = P.nz;
    GF_CU(klaunch<true>(eng, "k_em_fused", k_em_fused<S, R>, dim3(blocks_for((ny + 1) * (nz + 1), kThreads), (unsigned)(nx + 1)),
                  dim3(kThreads), 0, st, P, io, (int)eng->deck.mats.size(),
                  static_cast<const EmCls<R>*>(eng->em_cls_tab), eng->em_ncls));
    if (P.planeEM) GF_CU(klaunch(eng, "k_em_plane", k_em_plane<S, R>, dim3(blocks_for(nx * ny, kThreads)), dim3(kThreads), 0, st, P, io));
    if (!P.per_x) GF_CU(klaunch(eng, "k_em_mur_x", k_em_mur<S, 0, R>, dim3(blocks_for(ny * (nz + 1) + (ny + 1) * nz, kThreads)), dim3(kThreads), 0, st, P, io));
    if (!P.per_y) GF_CU(klaunch(eng, "k_em_mur_y", k_em_mur<S, 1, R>, dim3(blocks_for(nx * (nz + 1) + (nx + 1) * nz, kThreads)), dim3(kThreads), 0, st, P, io));
    if (!P.per_z) GF_CU(klaunch(eng, "k_em_mur_z", k_em_mur<S, 2, R>, dim3(blocks_for(nx * (ny + 1) + (nx + 1) * ny, kThreads)), dim3(kThreads), 0, st, P, io));
    if (P.pec) GF_CU(klaunch(eng, "k_em_pec", k_em_pec<S, R>, dim3(blocks_for((ny + 1) * (nz + 1), kThreads), (unsigned)(nx + 1)),
                             dim3(kThreads), 0, st, P, io));
    if (P.drude) GF_CU(klaunch(eng, "k_drude", k_drude<S, R>, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, st, P, io));
    return GF_OK;
}

template <int S, class R>
int enqueue_stage(gf_engine* eng, int parity) {
    const Params& P = eng->P;
    const StageIOT<R>& io = stage_io<R>(eng, parity, S);
    cudaStream_t st = eng->stream;
    const unsigned bn = blocks_for(P.n, kThreads);
    // The physics of a stage read only the stage inputs, except for these
    // dependencies: the LLG and (FP64) TDGL kernels read the cell strain the
    // elastic tile writes, flexoelectric runs read k_flexo_prep's arrays, the
    // Maxwell update reads the LLG increment (M-sourced current, spin
    // pumping), and the PEC kernel clears the step-start E that the TDGL
    // kernel reads at stage 1.  So the elastic chain runs on the engine
    // stream and the LLG, TDGL and Maxwell kernels on three branch streams
    // forked from it and joined before the static solves; the tiny boundary
    // kernels and the tails of the big ones then overlap other physics.
    // (per-kernel timing, gf_profile_steps, keeps one stream: each kernel is
    // then timed alone; so does a run with a single physics group, where a
    // fork would only add graph edges)
    const int groups = (P.elastic ? 1 : 0) + ((P.fm || P.afm) ? 1 : 0) + (P.fe ? 1 : 0) + (P.em ? 1 : 0);
    const bool par = !eng->profiling && groups >= 2;
    auto rec = [&](cudaEvent_t e, cudaStream_t s_) { return par ? cudaEventRecord(e, s_) : cudaSuccess; };
    auto wait_ = [&](cudaStream_t s_, cudaEvent_t e, unsigned) { return par ? cudaStreamWaitEvent(s_, e, 0) : cudaSuccess; };
    cudaStream_t s_llg = par ? eng->side[0] : st, s_fe = par ? eng->side[1] : st, s_em = par ? eng->side[2] : st;
    cudaEvent_t ev_start = eng->bev[0], ev_pre = eng->bev[1], ev_tile = eng->bev[2];
    cudaEvent_t ev_llg = eng->bev[3], ev_fe = eng->bev[4], ev_em = eng->bev[5];
    const bool mag = P.fm || P.afm;
    const bool em_after_llg = P.em && mag && (P.em_fromM || P.spin);
    const bool em_after_fe = P.em && P.fe && P.pec;
    const bool fe_after_tile = P.fe && P.elastic && P.elasto_on && !is_mixed<R>::value;
    GF_CU(rec(ev_start, st));
    if (P.em && !em_after_llg && !em_after_fe) {
        GF_CU(wait_(s_em, ev_start, 0));
        GF_TRY((enqueue_em<S, R>(eng, io, s_em)));
        GF_CU(rec(ev_em, s_em));
    }
    if (P.flexo)
        GF_CU(klaunch(eng, "k_flexo_prep", k_flexo_prep<R>, dim3(blocks_for((long)P.ny * P.nz, kThreads), (unsigned)P.nx),
                      dim3(kThreads), 0, st, P, io));
    GF_CU(rec(ev_pre, st));
    if (P.fe && !fe_after_tile) {
        GF_CU(wait_(s_fe, ev_pre, 0));
        GF_TRY((enqueue_fe<S, R>(eng, io, s_fe)));
        GF_CU(rec(ev_fe, s_fe));
    }
    if (P.elastic) {
        const dim3 grid((P.nz + etile::TK - 1) / etile::TK, (P.ny + etile::TJ - 1) / etile::TJ,
                        (P.nx + eng->el_chunk - 1) / eng->el_chunk);
        const ETileMaps& tm = eng->etm[parity][S];
        if (eng->el_cubic)
            GF_CU(klaunch<true>(eng, "k_elastic", k_elastic_tile<S, true, R>, grid, dim3(etile::NT), eng->el_smem, st, P, io,
                                eng->el_chunk, eng->el_nmat, tm));
        else
            GF_CU(klaunch<true>(eng, "k_elastic", k_elastic_tile<S, false, R>, grid, dim3(etile::NT), eng->el_smem, st, P, io,
                                eng->el_chunk, eng->el_nmat, tm));
    }
    GF_CU(rec(ev_tile, st));
    if (P.fe && fe_after_tile) {
        GF_CU(wait_(s_fe, ev_tile, 0));
        GF_TRY((enqueue_fe<S, R>(eng, io, s_fe)));
        GF_CU(rec(ev_fe, s_fe));
    }
    if (mag) {
        GF_CU(wait_(s_llg, ev_tile, 0));
        if (P.fm) GF_CU(klaunch<true>(eng, "k_llg_fm", k_llg_fm<S, R>, dim3(blocks_for(P.fm_bj * P.fm_bk, kThreads), (unsigned)P.fm_bi),
                                      dim3(kThreads), 0, s_llg, P, io, llg_tables<R>(eng), (int)eng->deck.mats.size()));
        if (P.afm) GF_CU(klaunch<true>(eng, "k_llg_afm", k_llg_afm<S, R>, dim3(blocks_for(P.afm_bj * P.afm_bk, kThreads), (unsigned)P.afm_bi),
                                       dim3(kThreads), 0, s_llg, P, io, llg_tables<R>(eng), (int)eng->deck.mats.size()));
        if (P.prescribed_m)
            GF_CU(klaunch(eng, "k_prescribed_m", k_prescribed_m<S, R>, dim3(blocks_for((long)P.nx * P.ny, kThreads)), dim3(kThreads), 0,
                          s_llg, P, io));
        GF_CU(rec(ev_llg, s_llg));
    }
    if (P.em && (em_after_llg || em_after_fe)) {
        if (em_after_llg) GF_CU(wait_(s_em, ev_llg, 0));
        if (em_after_fe) GF_CU(wait_(s_em, ev_fe, 0));
        GF_TRY((enqueue_em<S, R>(eng, io, s_em)));
        GF_CU(rec(ev_em, s_em));
    }
    if (P.elastic) {
        // the mixed form's RK kernel updates two cells per thread
        const unsigned brk = is_mixed<R>::value ? blocks_for(P.n, 2 * kThreads) : bn;
        GF_CU(klaunch(eng, "k_elastic_rk", k_elastic_rk<S, R>, dim3(brk), dim3(kThreads), 0, st, P, io));
        if (!P.el_bc_fused)
            GF_CU(klaunch(eng, "k_elastic_bc", k_elastic_bc<S, R>, dim3(blocks_for((long)P.nx * P.ny, kThreads)), dim3(kThreads), 0, st, P, io));
    }
    // join the branches
    if (mag) GF_CU(wait_(st, ev_llg, 0));
    if (P.fe) GF_CU(wait_(st, ev_fe, 0));
    if (P.em) GF_CU(wait_(st, ev_em, 0));
    if (eng->demag_per_stage) {
        // static field of the new stage state (main.cpp:299-306, 476-483)
        if constexpr (is_mixed<R>::value) GF_TRY(demag_solve_f32(eng, io.m_out, io.a1_out, io.a2_out, true, io.msrc != nullptr));
        else GF_TRY(demag_solve(eng, io.m_out, io.a1_out, io.a2_out, true, io.msrc != nullptr));
    }
    if (eng->elec_on && eng->elec_per_stage) {
        // electrostatic field of the new stage polarisation (main.cpp:299-302;
        // the 1-D model after every p update, ferroelectric_solver.cpp:1897-1990)
        if (eng->elec_1d) {
            GF_CU(klaunch(eng, "k_elec_1d", k_elec_1d<R>, dim3(blocks_for((long)P.nx * P.ny, kThreads)), dim3(kThreads), 0, st,
                          P, io.mats, io.mid, (const R*)io.p_out.c[2], (const R*)reinterpret_cast<R*>(eng->elec_pz_t0), io.Estat));
        } else if constexpr (!is_mixed<R>::value) {
            GF_TRY(elec_solve(eng, io.p_out, true, eng->elec_iters, 0., nullptr));
        }
    }
    return GF_OK;
}

// Mean device time of `reps` launches of the stage-1 elastic tile kernel at
// the engine's current x-chunk.  The kernel writes only per-stage scratch (the
// stress divergence and the cell strain), so timing it leaves the state alone.
template <class R>
int time_tile_t(gf_engine* eng, int reps, float* ms) {
    const Params& P = eng->P;
    const StageIOT<R>& io = stage_io<R>(eng, (int)(eng->steps_done & 1ull), 0);
    const dim3 grid((P.nz + etile::TK - 1) / etile::TK, (P.ny + etile::TJ - 1) / etile::TJ,
                    (P.nx + eng->el_chunk - 1) / eng->el_chunk);
    cudaEvent_t a, b;
    GF_CU(cudaEventCreate(&a));
    GF_CU(cudaEventCreate(&b));
    const ETileMaps& tm = eng->etm[(int)(eng->steps_done & 1ull)][0];
    auto one = [&]() {
        return eng->el_cubic ? launch_tiled(k_elastic_tile<0, true, R>, grid, dim3(etile::NT), eng->el_smem, eng->stream, P, io,
                                            eng->el_chunk, eng->el_nmat, tm)
                             : launch_tiled(k_elastic_tile<0, false, R>, grid, dim3(etile::NT), eng->el_smem, eng->stream, P, io,
                                            eng->el_chunk, eng->el_nmat, tm);
    };
    cudaError_t e = one();                     // warm
    if (e == cudaSuccess) e = cudaEventRecord(a, eng->stream);
    for (int r = 0; r < reps && e == cudaSuccess; r++) e = one();
    if (e == cudaSuccess) e = cudaEventRecord(b, eng->stream);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    GF_CU(e);
    *ms = t / (float)(reps > 0 ? reps : 1);
    return GF_OK;
}

template <class R>
int enqueue_step_t(gf_engine* eng, int parity) {
    GF_TRY((enqueue_stage<0, R>(eng, parity)));
    GF_TRY((enqueue_stage<1, R>(eng, parity)));
    GF_TRY((enqueue_stage<2, R>(eng, parity)));
    GF_TRY((enqueue_stage<3, R>(eng, parity)));
    return GF_OK;
}

}  // namespace

template <class R>
int enqueue_stage_t(gf_engine* eng, int parity, int s) {
    if (s == 0) return enqueue_stage<0, R>(eng, parity);
    if (s == 1) return enqueue_stage<1, R>(eng, parity);
    if (s == 2) return enqueue_stage<2, R>(eng, parity);
    return enqueue_stage<3, R>(eng, parity);
}

#ifdef GF_MIXED_TU
int gf_mixed_enqueue_step(gf_engine* eng, int parity) { return enqueue_step_t<float>(eng, parity); }
int gf_mixed_enqueue_stage(gf_engine* eng, int parity, int s) { return enqueue_stage_t<float>(eng, parity, s); }

int gf_mixed_elastic_setup(gf_engine* eng, int smem, int* per_sm) {
    GF_TRY(set_elastic_smem<float>(eng, smem));
    GF_CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_elastic_tile<1, false, float>, etile::NT, (size_t)smem));
    return GF_OK;
}

int gf_mixed_time_tile(gf_engine* eng, int reps, float* ms) { return time_tile_t<float>(eng, reps, ms); }

// the FP32 elastic tile (rk = 0) or RK update (rk = 1) of stage s on the
// discrete adjoint's buffers (io built by the adjoint), with the engine's
// launch shapes; the tile stages by cp.async (no tensor maps over the
// adjoint's buffers)
namespace {
template <int S>
int adj_elastic_f32(gf_engine* eng, int rk, const StageIOT<float>& io) {
    const Params& P = eng->P;
    if (rk) {
        // the adjoint applies the Liao boundary itself, after the step
        Params Pa = P;
        Pa.el_bc_fused = 0;
        GF_CU(launch(k_elastic_rk<S, float>, dim3(blocks_for(P.n, 2 * kThreads)), dim3(kThreads), 0, eng->stream, Pa, io));
        return GF_OK;
    }
    ETileMaps tm;
    std::memset(&tm, 0, sizeof(tm));
    tm.err = eng->tma_err;
    const dim3 grid((P.nz + etile::TK - 1) / etile::TK, (P.ny + etile::TJ - 1) / etile::TJ,
                    (P.nx + eng->el_chunk - 1) / eng->el_chunk);
    if (eng->el_cubic)
        GF_CU(launch_tiled(k_elastic_tile<S, true, float>, grid, dim3(etile::NT), eng->el_smem, eng->stream, P, io,
                           eng->el_chunk, eng->el_nmat, tm));
    else
        GF_CU(launch_tiled(k_elastic_tile<S, false, float>, grid, dim3(etile::NT), eng->el_smem, eng->stream, P, io,
                           eng->el_chunk, eng->el_nmat, tm));
    return GF_OK;
}
}  // namespace

int gf_mixed_batch_attr(size_t smem) {
    const int b = (int)smem;
    cudaError_t e = cudaSuccess;
    auto set = [&](auto k) { if (e == cudaSuccess) e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, b); };
    set(k_batch_phase<0, 0>); set(k_batch_phase<1, 0>); set(k_batch_phase<2, 0>); set(k_batch_phase<3, 0>);
    set(k_batch_phase<0, 3>); set(k_batch_phase<1, 3>); set(k_batch_phase<2, 3>); set(k_batch_phase<3, 3>);
    set(k_batch_persistent);
    return e == cudaSuccess ? GF_OK : GF_ECUDA;
}

int gf_mixed_batch_persistent_blocks(size_t smem, int* blocks) {
    int per = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_persistent, 256, smem) != cudaSuccess) return GF_ECUDA;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return GF_ECUDA;
    *blocks = per * sms;
    return GF_OK;
}

// one cooperative launch (every block resident) of the persistent step
int gf_mixed_batch_persistent(const BatchInst* insts, int ninst, const BatchItem* A, int nA, const BatchItem* L, int nB, int nC,
                              int nD, int parity, size_t smem, unsigned* err, unsigned* bar, int blocks, cudaStream_t st) {
    ETileMaps tm;
    std::memset(&tm, 0, sizeof(tm));
    tm.err = err;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)blocks);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return (int)cudaLaunchKernelEx(&cfg, k_batch_persistent, insts, ninst, A, nA, L, nB, nC, nD, parity, tm, bar);
}

int gf_mixed_batch_phase(const BatchInst* insts, const BatchItem* items, int count, int s, int ph, int parity, size_t smem,
                         unsigned* tma_err, cudaStream_t st) {
    if (count <= 0) return (int)cudaSuccess;
    ETileMaps tm;
    std::memset(&tm, 0, sizeof(tm));
    tm.err = tma_err;
    const dim3 g((unsigned)count), b(256);
    const size_t em_tab = kMaxMat * sizeof(EmMat<float>) + kEmMaxCls * sizeof(EmCls<float>);
    const size_t sm = (ph == 0 || ph == 3) ? smem : (ph == 4 ? em_tab : 0);
    cudaError_t e = cudaErrorInvalidValue;
#define GF_BPH(S_, P_) if (s == S_ && ph == P_) e = launch(k_batch_phase<S_, P_>, g, b, sm, st, insts, items, parity, tm)
    GF_BPH(0, 0); GF_BPH(0, 1); GF_BPH(1, 0); GF_BPH(1, 1);
    GF_BPH(2, 0); GF_BPH(2, 1); GF_BPH(3, 0); GF_BPH(3, 1);
    GF_BPH(0, 3); GF_BPH(0, 4); GF_BPH(0, 5); GF_BPH(1, 3); GF_BPH(1, 4); GF_BPH(1, 5);
    GF_BPH(2, 3); GF_BPH(2, 4); GF_BPH(2, 5); GF_BPH(3, 3); GF_BPH(3, 4); GF_BPH(3, 5);
#undef GF_BPH
    return (int)e;
}

int gf_mixed_adj_elastic(gf_engine* eng, int s, int rk, const StageIOT<float>& io) {
    if (s == 0) return adj_elastic_f32<0>(eng, rk, io);
    if (s == 1) return adj_elastic_f32<1>(eng, rk, io);
    if (s == 2) return adj_elastic_f32<2>(eng, rk, io);
    return adj_elastic_f32<3>(eng, rk, io);
}
#else
namespace {

int es_solve(gf_engine* eng, int parity, bool counted, int iters, double tol, int* used);
int elec_1d_now(gf_engine* eng, int parity);

// work after the fourth stage: the elastostatic solve of the new state when
// it runs without elastodynamics (main.cpp:472-474)
int step_end(gf_engine* eng, int parity, bool counted) {
    if (eng->es_on && eng->es_per_step) GF_TRY(es_solve(eng, 1 - parity, counted, eng->es_iters, 0., nullptr));
    return GF_OK;
}

int enqueue_step(gf_engine* eng, int parity) {
    eng->launch_counter = 0;
    if (eng->mixed) GF_TRY(gf_mixed_enqueue_step(eng, parity));
    else GF_TRY(enqueue_step_t<double>(eng, parity));
    GF_TRY(step_end(eng, parity, true));
    GF_CU(klaunch(eng, "k_step_inc", k_step_inc, dim3(1), dim3(1), 0, eng->stream, eng->step_ctr));
    eng->launches_per_step = eng->launch_counter;
    return GF_OK;
}

// static field from the current m (initial solve, main.cpp:135-146)
int static_field_now(gf_engine* eng) {
    if (eng->demag_mode < 0) return GF_OK;
    if (eng->mixed) return demag_solve_f32(eng, f3f(eng->m.X), f3f(eng->a1.X), f3f(eng->a2.X), false);
    return demag_solve(eng, f3(eng->m.X), f3(eng->a1.X), f3(eng->a2.X), false);
}

// The nine demag tensor tables (9 x n, table-major) of a grid, built on the
// host with the host's libm on all cores: the reference builds them on the
// host too (initialize_intermediate_Hms), and the far-field entries are small
// differences of large terms, so a last-bit difference in log or atan would
// grow by orders of magnitude there.  The last grid's tables are kept, so an
// FP64 and a mixed engine of the same deck build them once.
std::shared_ptr<const std::vector<double>> newell_tables(const Params& P) {
    static std::mutex mu;
    static std::shared_ptr<const std::vector<double>> last;
    static double key[6] = {0, 0, 0, 0, 0, 0};
    const double k6[6] = {(double)P.nx, (double)P.ny, (double)P.nz, P.dx, P.dy, P.dz};
    std::lock_guard<std::mutex> lock(mu);
    if (last && std::memcmp(key, k6, sizeof(k6)) == 0) return last;
    auto tab = std::make_shared<std::vector<double>>((size_t)9 * P.n);
    double* out = tab->data();
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt == 0 ? 1 : (nt > 64 ? 64 : nt);
    const long n = P.n;
    auto work = [&](unsigned w) {
        double v[9];
        for (long c = w; c < n; c += nt) {
            newell_cell(P, c, v);
            for (int t = 0; t < 9; t++) out[(size_t)t * n + c] = v[t];
        }
    };
    std::vector<std::thread> th;
    for (unsigned w = 1; w < nt; w++) th.emplace_back(work, w);
    work(0);
    for (auto& x : th) x.join();
    last = tab;
    std::memcpy(key, k6, sizeof(k6));
    return last;
}

int setup_demag(gf_engine* eng) {
    const Deck& d = eng->deck;
    const Params& P = eng->P;
    if (!(d.any_fm || d.any_afm) || !d.magnetostatics) { eng->demag_mode = -1; return GF_OK; }
    if (d.mag_1D) eng->demag_mode = 2;
    else if (d.demag_factor) eng->demag_mode = 1;
    else eng->demag_mode = 0;
    eng->demag_per_stage = !d.em_dynamic;
    // the LLG kernel can form the per-stage transform input itself when it
    // visits every cell (the ferromagnet's bounding box is the grid) and no
    // antiferromagnet adds to M
    eng->demag_src_fused = eng->demag_per_stage && !d.mag_1D && !d.demag_factor && P.fm && !P.afm &&
                           P.fm_bi * P.fm_bj * P.fm_bk == P.n && !P.prescribed_m;
    if (eng->demag_mode != 0) return GF_OK;
    const long n21 = (long)P.nx * P.ny * (P.nz / 2 + 1);
    int dims[3] = {P.nx, P.ny, P.nz};
    if (eng->mixed) {
        // M (3n real), M_k (3 n21 complex) and the six real spectra in FP32
        GF_TRY(dalloc(eng, reinterpret_cast<void**>(&eng->Mfft), sizeof(float) * 3 * (size_t)P.n));
        GF_TRY(dalloc(eng, reinterpret_cast<void**>(&eng->Mk), sizeof(cufftComplex) * 3 * (size_t)n21));
        GF_TRY(dalloc(eng, reinterpret_cast<void**>(&eng->Nr), sizeof(float) * 6 * (size_t)n21));
        // tables and their spectra in FP64 with a temporary D2Z plan, then rounded to FP32
        double* tab = nullptr;
        cufftDoubleComplex* nk64 = nullptr;
        cufftHandle p64 = 0;
        const std::shared_ptr<const std::vector<double>> host_tab = newell_tables(P);
        cudaError_t ce = cudaMalloc(&tab, sizeof(double) * 9 * (size_t)P.n);
        if (ce == cudaSuccess) ce = cudaMalloc(&nk64, sizeof(cufftDoubleComplex) * 9 * (size_t)n21);
        cufftResult fr = CUFFT_SUCCESS;
        if (ce == cudaSuccess) fr = cufftPlanMany(&p64, 3, dims, nullptr, 1, (int)P.n, nullptr, 1, (int)n21, CUFFT_D2Z, 3);
        if (ce == cudaSuccess && fr == CUFFT_SUCCESS) fr = cufftSetStream(p64, eng->stream);
        if (ce == cudaSuccess && fr == CUFFT_SUCCESS)
            ce = cudaMemcpyAsync(tab, host_tab->data(), sizeof(double) * 9 * (size_t)P.n, cudaMemcpyHostToDevice, eng->stream);
        for (int b = 0; b < 3 && ce == cudaSuccess && fr == CUFFT_SUCCESS; b++)
            fr = cufftExecD2Z(p64, tab + (size_t)3 * b * P.n, nk64 + (size_t)3 * b * n21);
        if (ce == cudaSuccess && fr == CUFFT_SUCCESS)
            ce = launch(k_spectra_real<float>, dim3(blocks_for(n21, kThreads)), dim3(kThreads), 0, eng->stream,
                        (const cuDoubleComplex*)nk64, n21, eng->Nr);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(eng->stream);
        if (p64) cufftDestroy(p64);
        if (tab) cudaFree(tab);
        if (nk64) cudaFree(nk64);
        if (ce != cudaSuccess) { eng->err = std::string("demag tables: ") + cudaGetErrorString(ce); return GF_ECUDA; }
        if (fr != CUFFT_SUCCESS) { eng->err = "demag tables: cuFFT error " + std::to_string((int)fr); return GF_ECUDA; }
        GF_FFT(cufftPlanMany(&eng->plan_r2c, 3, dims, nullptr, 1, (int)P.n, nullptr, 1, (int)n21, CUFFT_R2C, 3));
        GF_FFT(cufftPlanMany(&eng->plan_c2r, 3, dims, nullptr, 1, (int)n21, nullptr, 1, (int)P.n, CUFFT_C2R, 3));
        eng->plans = true;
        GF_FFT(cufftSetStream(eng->plan_r2c, eng->stream));
        GF_FFT(cufftSetStream(eng->plan_c2r, eng->stream));
        for (int a = 0; a < 3; a++) eng->Hstat[a] = reinterpret_cast<double*>(reinterpret_cast<float*>(eng->Mfft) + (size_t)a * P.n);
        return GF_OK;
    }
    GF_TRY(dalloc_n(eng, &eng->Mfft, (size_t)3 * P.n));
    GF_TRY(dalloc_n(eng, &eng->Mk, (size_t)3 * n21));
    GF_TRY(dalloc_n(eng, &eng->Nk, (size_t)9 * n21));
    // H_stat is a view of the FFT buffer: the inverse transform writes it,
    // and the next stage's source overwrites it only after the LLG kernels
    // of that stage have read it
    for (int a = 0; a < 3; a++) eng->Hstat[a] = eng->Mfft + (size_t)a * P.n;
    GF_FFT(cufftPlanMany(&eng->plan_r2c, 3, dims, nullptr, 1, (int)P.n, nullptr, 1, (int)n21, CUFFT_D2Z, 3));
    GF_FFT(cufftPlanMany(&eng->plan_c2r, 3, dims, nullptr, 1, (int)n21, nullptr, 1, (int)P.n, CUFFT_Z2D, 3));
    eng->plans = true;
    GF_FFT(cufftSetStream(eng->plan_r2c, eng->stream));
    GF_FFT(cufftSetStream(eng->plan_c2r, eng->stream));
    // demag tensor tables: 9 x n real, built on the host, transformed on the
    // device in three batches of 3
    const std::shared_ptr<const std::vector<double>> host_tab = newell_tables(P);
    double* tab = nullptr;                                                    // temporary
    cudaError_t ce = cudaMalloc(&tab, sizeof(double) * 9 * (size_t)P.n);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(tab, host_tab->data(), sizeof(double) * 9 * (size_t)P.n, cudaMemcpyHostToDevice, eng->stream);
    cufftResult fr = CUFFT_SUCCESS;
    for (int b = 0; b < 3 && ce == cudaSuccess && fr == CUFFT_SUCCESS; b++)
        fr = cufftExecD2Z(eng->plan_r2c, tab + (size_t)3 * b * P.n, eng->Nk + (size_t)3 * b * n21);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(eng->stream);
    if (tab) cudaFree(tab);
    if (ce != cudaSuccess) { eng->err = std::string("demag tables: ") + cudaGetErrorString(ce); return GF_ECUDA; }
    if (fr != CUFFT_SUCCESS) { eng->err = "demag tables: cuFFT error " + std::to_string((int)fr); return GF_ECUDA; }
    return GF_OK;
}

// one host FP64 array into a device buffer of the run's precision; in the
// mixed form the value is split into an FP32 value and, when `cmp` is given,
// its FP32 rounding error (the compensation word)
int upload_one(gf_engine* eng, double* dst, double* cmp, const double* src, long n) {
    if (!eng->mixed) {
        GF_CU(cudaMemcpy(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice));
        return GF_OK;
    }
    std::vector<float> hi((size_t)n), lo(cmp ? (size_t)n : 0);
    for (long i = 0; i < n; i++) {
        hi[(size_t)i] = (float)src[i];
        if (cmp) lo[(size_t)i] = (float)(src[i] - (double)hi[(size_t)i]);
    }
    GF_CU(cudaMemcpy(dst, hi.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    if (cmp) GF_CU(cudaMemcpy(cmp, lo.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    return GF_OK;
}

int upload_vec(gf_engine* eng, double* const* dst, const std::vector<double>* src, long n, double* const* cmp = nullptr) {
    GF_CU(cudaStreamSynchronize(eng->stream));
    for (int a = 0; a < 3; a++) GF_TRY(upload_one(eng, dst[a], cmp ? cmp[a] : nullptr, src[a].data(), n));
    return GF_OK;
}

// copy the current-step buffer of every state field into its other three
// buffers, so cells a stage kernel does not cover stay consistent
int replicate_state(gf_engine* eng) {
    Field3* fs[] = {&eng->m, &eng->a1, &eng->a2, &eng->p, &eng->q, &eng->u, &eng->v, &eng->E, &eng->H,
                    &eng->jp[0], &eng->jp[1], &eng->jp[2]};
    for (Field3* f : fs) {
        if (!f->on) continue;
        double* const* c = (eng->steps_done & 1ull) ? f->A : f->X;
        for (int a = 0; a < 3; a++) {
            double* others[3] = {(c == f->A) ? f->X[a] : f->A[a], f->S0[a], f->S1[a]};
            for (double* o : others)
                GF_CU(cudaMemcpyAsync(o, c[a], eng->esz * f->len[a], cudaMemcpyDeviceToDevice, eng->stream));
        }
    }
    GF_CU(cudaStreamSynchronize(eng->stream));
    return GF_OK;
}

// out = Tg2c in Tg2c^T with the loop and rounding order of
// transform_matrix_glb2crt (mathlib.cpp:78-100); a copy without rotation
void glb2crt_tensor_host(const Deck& d, const double in[3][3], double out[3][3]) {
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            if (!d.orient_rotate) { out[i][j] = in[i][j]; continue; }
            out[i][j] = 0.;
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) out[i][j] = out[i][j] + d.Tg2c[i][k] * d.Tg2c[j][l] * in[k][l];
        }
}

// Static strain (strain_stat.in: global frame, rotated to the crystal frame
// with vacuum cells at zero, elastic_initialize.cpp:424-455) and static
// eigenstrain (eigenstraint0_crt.in: crystal frame as read) of
// inoutput.cpp:239-280
int read_static_strain(gf_engine* eng, const std::string& dir) {
    const Deck& d = eng->deck;
    const long n = d.n();
    std::vector<double> b6[6];
    for (auto& b : b6) b.assign((size_t)n, 0.);
    if (d.in_straint0) {
        std::string e = read_restart(dir + "/strain_stat.in", d.nx, d.ny, d.nz, 6, b6);
        if (!e.empty()) { eng->err = e; return GF_EIO; }
        for (long c = 0; c < n; c++) {
            const size_t u = (size_t)c;
            if (d.material_cell[u] == 0) { for (auto& b : b6) b[u] = 0.; continue; }
            const double in[3][3] = {{b6[0][u], b6[5][u], b6[4][u]}, {b6[5][u], b6[1][u], b6[3][u]}, {b6[4][u], b6[3][u], b6[2][u]}};
            double out[3][3];
            glb2crt_tensor_host(d, in, out);
            b6[0][u] = out[0][0]; b6[1][u] = out[1][1]; b6[2][u] = out[2][2];
            b6[3][u] = out[1][2]; b6[4][u] = out[0][2]; b6[5][u] = out[0][1];
        }
        for (int a = 0; a < 6; a++) {
            GF_TRY(dalloc_r(eng, &eng->es_eps[a], (size_t)n));
            GF_TRY(upload_one(eng, eng->es_eps[a], nullptr, b6[a].data(), n));
        }
    }
    if (d.in_eig0) {
        for (auto& b : b6) std::fill(b.begin(), b.end(), 0.);
        std::string e = read_restart(dir + "/eigenstraint0_crt.in", d.nx, d.ny, d.nz, 6, b6);
        if (!e.empty()) { eng->err = e; return GF_EIO; }
        for (int a = 0; a < 6; a++) {
            GF_TRY(dalloc_r(eng, &eng->es_eig[a], (size_t)n));
            GF_TRY(upload_one(eng, eng->es_eig[a], nullptr, b6[a].data(), n));
        }
    }
    return GF_OK;
}

int initial_state(gf_engine* eng, const std::string& dir) {
    const Deck& d = eng->deck;
    const long n = d.n();
    const double PI = kPi;
    std::vector<double> buf[3];
    for (auto& b : buf) b.assign((size_t)n, 0.);
    if (eng->m.on) {
        if (d.in_m) {
            std::string e = read_restart(dir + "/m.in", d.nx, d.ny, d.nz, 3, buf);
            if (!e.empty()) { eng->err = e; return GF_EIO; }
        } else {
            // initialize_magnetization (magnetic_initialize.cpp:1131-1151)
            const double theta = (d.theta_mag) / 180. * PI;
            const double phi = (d.phi_mag) / 180 * PI;
            const double mx = std::sin(theta) * std::cos(phi), my = std::sin(theta) * std::sin(phi), mz = std::cos(theta);
            for (long c = 0; c < n; c++) {
                uint8_t id = d.material_cell[(size_t)c];
                if (id && d.mats[id - 1].fm) { buf[0][c] = mx; buf[1][c] = my; buf[2][c] = mz; }
            }
        }
        if (d.prescribed_m) {
            // initialize_device's update_prescribed_m at time 0
            // (magnetic_initialize.cpp:1072-1078): k = 0 ferromagnetic cells
            const double m0 = std::sin(d.precess_angle / 180. * PI);
            const double omega = 2. * PI * d.precess_freq;
            const double t0 = 0.;
            for (long i = 0; i < d.nx; i++)
                for (long j = 0; j < d.ny; j++) {
                    const long c = (i * d.ny + j) * d.nz;
                    const uint8_t id = d.material_cell[(size_t)c];
                    if (!(id && d.mats[id - 1].fm)) continue;
                    buf[0][c] = std::sqrt((1. - m0 * m0));
                    buf[1][c] = m0 * std::sin(omega * t0);
                    buf[2][c] = m0 * std::cos(omega * t0);
                }
        }
        GF_TRY(upload_vec(eng, eng->m.X, buf, n, eng->m.C));
    }
    if (eng->a1.on) {
        std::vector<double> b6[6];
        for (auto& b : b6) b.assign((size_t)n, 0.);
        if (d.in_afm) {
            // input_AFMm (inoutput.cpp:29-50): "i j k m1x m1y m1z m2x m2y m2z"
            std::string e = read_restart(dir + "/m_AFM.in", d.nx, d.ny, d.nz, 6, b6);
            if (!e.empty()) { eng->err = e; return GF_EIO; }
        } else {
            // initialize_magnetization_AFM (magnetic_initialize.cpp:1153-1174): m2 = -m1
            const double theta = (d.theta_mag) / 180. * PI;
            const double phi = (d.phi_mag) / 180 * PI;
            const double mx = std::sin(theta) * std::cos(phi), my = std::sin(theta) * std::sin(phi), mz = std::cos(theta);
            for (long c = 0; c < n; c++) {
                uint8_t id = d.material_cell[(size_t)c];
                if (id && d.mats[id - 1].afm) {
                    b6[0][c] = mx; b6[1][c] = my; b6[2][c] = mz;
                    b6[3][c] = -mx; b6[4][c] = -my; b6[5][c] = -mz;
                }
            }
        }
        GF_TRY(upload_vec(eng, eng->a1.X, b6, n, eng->a1.C));
        GF_TRY(upload_vec(eng, eng->a2.X, b6 + 3, n, eng->a2.C));
    }
    if (eng->p.on) {
        for (auto& b : buf) std::fill(b.begin(), b.end(), 0.);
        std::vector<double> qb[3];
        for (auto& b : qb) b.assign((size_t)n, 0.);
        if (d.in_pq) {
            std::string e = read_restart(dir + "/p.in", d.nx, d.ny, d.nz, 3, buf);
            if (e.empty()) e = read_restart(dir + "/q.in", d.nx, d.ny, d.nz, 3, qb);
            if (!e.empty()) { eng->err = e; return GF_EIO; }
        } else {
            for (long c = 0; c < n; c++) {
                uint8_t id = d.material_cell[(size_t)c];
                if (id && d.mats[id - 1].fe) { buf[0][c] = d.px_init; buf[1][c] = d.py_init; buf[2][c] = d.pz_init; }
            }
        }
        GF_TRY(upload_vec(eng, eng->p.X, buf, n, eng->p.C));
        GF_TRY(upload_vec(eng, eng->q.X, qb, n, eng->q.C));
    }
    if (eng->u.on && d.in_uv) {
        std::vector<double> ub[3], vb[3];
        for (auto& b : ub) b.assign((size_t)n, 0.);
        for (auto& b : vb) b.assign((size_t)n, 0.);
        std::string e = read_restart(dir + "/u.in", d.nx, d.ny, d.nz, 3, ub);
        if (e.empty()) e = read_restart(dir + "/v.in", d.nx, d.ny, d.nz, 3, vb);
        if (!e.empty()) { eng->err = e; return GF_EIO; }
        GF_TRY(upload_vec(eng, eng->u.X, ub, n, eng->u.C));
        GF_TRY(upload_vec(eng, eng->v.X, vb, n, eng->v.C));
    }
    if (d.in_force && eng->force_store[0]) {
        // elastoforce.in: the stage-1 stress divergence the next step's
        // stiffness damping reads (inoutput.cpp:220-237)
        for (auto& b : buf) std::fill(b.begin(), b.end(), 0.);
        std::string e = read_restart(dir + "/elastoforce.in", d.nx, d.ny, d.nz, 3, buf);
        if (!e.empty()) { eng->err = e; return GF_EIO; }
        GF_TRY(upload_vec(eng, eng->force_store, buf, n));
    }
    if (d.in_Jp) {
        // Jp1.in..Jp3.in: the Drude pole currents (inoutput.cpp:283-328)
        const char* names[3] = {"Jp1.in", "Jp2.in", "Jp3.in"};
        for (int pole = 0; pole < 3; pole++) {
            if (!eng->jp[pole].on) continue;
            for (auto& b : buf) std::fill(b.begin(), b.end(), 0.);
            std::string e = read_restart(dir + "/" + names[pole], d.nx, d.ny, d.nz, 3, buf);
            if (!e.empty()) { eng->err = e; return GF_EIO; }
            GF_TRY(upload_vec(eng, eng->jp[pole].X, buf, n, eng->jp[pole].C));
        }
    }
    if (eng->E.on && d.in_em) {
        const char* names[6] = {"Ex_Yee.in", "Ey_Yee.in", "Ez_Yee.in", "Hx_Yee.in", "Hy_Yee.in", "Hz_Yee.in"};
        for (int f = 0; f < 6; f++) {
            const Field3& F = f < 3 ? eng->E : eng->H;
            const int c = f % 3;
            long dimx = d.nx, dimy = d.ny, dimz = d.nz;
            if (f < 3) { dimx += (c != 0); dimy += (c != 1); dimz += (c != 2); }
            else { dimx += (c == 0); dimy += (c == 1); dimz += (c == 2); }
            std::vector<double> one((size_t)(dimx * dimy * dimz), 0.);
            std::string e = read_restart(dir + "/" + names[f], dimx, dimy, dimz, 1, &one);
            if (!e.empty()) { eng->err = e; return GF_EIO; }
            GF_TRY(upload_one(eng, F.X[c], F.C[c], one.data(), (long)one.size()));
        }
    }
    if (d.in_Hstat && eng->Hstat[0]) {
        for (auto& b : buf) std::fill(b.begin(), b.end(), 0.);
        std::string e = read_restart(dir + "/Hstat.in", d.nx, d.ny, d.nz, 3, buf);
        if (!e.empty()) { eng->err = e; return GF_EIO; }
        GF_TRY(upload_vec(eng, eng->Hstat, buf, n));
    }
    if (d.in_Estat && eng->Estat[0]) {
        for (auto& b : buf) std::fill(b.begin(), b.end(), 0.);
        std::string e = read_restart(dir + "/Estat.in", d.nx, d.ny, d.nz, 3, buf);
        if (!e.empty()) { eng->err = e; return GF_EIO; }
        GF_TRY(upload_vec(eng, eng->Estat, buf, n));
        eng->P.estat = 1;
    }
    if (d.read_Hext_nonunif) {
        for (auto& b : buf) std::fill(b.begin(), b.end(), 0.);
        std::string e = read_restart(dir + "/Hext_nonunif.in", d.nx, d.ny, d.nz, 3, buf);
        if (!e.empty()) { eng->err = e; return GF_EIO; }
        GF_TRY(upload_vec(eng, eng->Hnu, buf, n));
    }
    if (d.in_straint0 || d.in_eig0) GF_TRY(read_static_strain(eng, dir));
    return GF_OK;
}

// Material class of the E edge whose four cells (in the kernel's order 1..4)
// hold ids[]: the kernel's sums and division, done here once per class.
template <class R>
EmCls<R> em_class(const Deck& d, const unsigned ids[4], R dt_e0) {
    R er = R(0.), cond = R(0.), pc = R(0.);
    uint32_t mask = 0;
    for (int q = 0; q < 4; q++) {
        if (ids[q] == 0) { er = er + R(1.); continue; }
        const Material& m = d.mats[ids[q] - 1];
        mask |= 1u << q;
        if (m.fe) pc = pc + R(1.);
        er = er + static_cast<R>(m.er);
        cond = cond + static_cast<R>(m.cond);
    }
    if (pc < R(0.5)) pc = R(1.);
    er = er / R(4.);
    EmCls<R> c;
    c.coef = dt_e0 / er;
    c.cond = cond / R(4.);
    c.pc = pc;
    c.mask = mask;
    c.pad_ = 0;
    return c;
}

// Per-edge classes of the Yee E update (k_em_fused): one byte per edge and a
// table of the distinct cell quadruples.  A deck with more quadruples than a
// byte indexes keeps the per-cell material lookups (Params::em_cls = 0).
// Edges on a non-periodic boundary are not updated by that kernel; they get
// class 0.
int setup_em_classes(gf_engine* eng) {
    Params& P = eng->P;
    const Deck& d = eng->deck;
    const long nx = P.nx, ny = P.ny, nz = P.nz;
    auto mc = [&](long i, long j, long k) -> unsigned { return d.material_cell[(size_t)((i * ny + j) * nz + k)]; };
    // class of each quadruple of ids 0..kMaxMat, -1 until first seen
    constexpr int K = kMaxMat + 1;
    std::vector<int> index((size_t)K * K * K * K, -1);
    std::vector<uint32_t> keys;
    std::vector<uint8_t> cls[3];
    const long ext[3][3] = {{nx, ny + 1, nz + 1}, {nx + 1, ny, nz + 1}, {nx + 1, ny + 1, nz}};
    // neighbour cells of a node coordinate along an axis of n cells: (lower, upper), wrapped at the ends
    auto lo = [](long c, long n) { return (c == 0 || c == n) ? n - 1 : c - 1; };
    auto hi = [](long c, long n) { return (c == 0 || c == n) ? 0 : c; };
    for (int C = 0; C < 3; C++) {
        cls[C].assign((size_t)(ext[C][0] * ext[C][1] * ext[C][2]), 0);
        for (long i = 0; i < ext[C][0]; i++)
            for (long j = 0; j < ext[C][1]; j++)
                for (long k = 0; k < ext[C][2]; k++) {
                    bool bnd = false;
                    unsigned ids[4];
                    if (C == 0) {
                        bnd = ((j == 0 || j == ny) && !P.per_y) || ((k == 0 || k == nz) && !P.per_z);
                        const long y1 = lo(j, ny), y3 = hi(j, ny), z1 = lo(k, nz), z2 = hi(k, nz);
                        ids[0] = mc(i, y1, z1); ids[1] = mc(i, y1, z2); ids[2] = mc(i, y3, z1); ids[3] = mc(i, y3, z2);
                    } else if (C == 1) {
                        bnd = ((i == 0 || i == nx) && !P.per_x) || ((k == 0 || k == nz) && !P.per_z);
                        const long x1 = lo(i, nx), x3 = hi(i, nx), z1 = lo(k, nz), z2 = hi(k, nz);
                        ids[0] = mc(x1, j, z1); ids[1] = mc(x1, j, z2); ids[2] = mc(x3, j, z1); ids[3] = mc(x3, j, z2);
                    } else {
                        bnd = ((i == 0 || i == nx) && !P.per_x) || ((j == 0 || j == ny) && !P.per_y);
                        const long x1 = lo(i, nx), x3 = hi(i, nx), y1 = lo(j, ny), y2 = hi(j, ny);
                        ids[0] = mc(x1, y1, k); ids[1] = mc(x1, y2, k); ids[2] = mc(x3, y1, k); ids[3] = mc(x3, y2, k);
                    }
                    if (bnd) continue;
                    const uint32_t key = ids[0] | (ids[1] << 8) | (ids[2] << 16) | (ids[3] << 24);
                    int& c = index[(((size_t)ids[0] * K + ids[1]) * K + ids[2]) * K + ids[3]];
                    if (c < 0) {
                        if ((int)keys.size() >= kEmMaxCls) { P.em_cls = 0; return GF_OK; }
                        c = (int)keys.size();
                        keys.push_back(key);
                    }
                    cls[C][(size_t)((i * ext[C][1] + j) * ext[C][2] + k)] = (uint8_t)c;
                }
    }
    if (keys.empty()) keys.push_back(0u);
    const size_t nk = keys.size();
    auto ids_of = [](uint32_t key, unsigned* ids) { for (int q = 0; q < 4; q++) ids[q] = (key >> (8 * q)) & 0xffu; };
    if (eng->mixed) {
        std::vector<EmCls<float>> t(nk);
        for (size_t c = 0; c < nk; c++) { unsigned ids[4]; ids_of(keys[c], ids); t[c] = em_class<float>(d, ids, P.f.dt_e0); }
        EmCls<float>* dp = nullptr;
        GF_TRY(dalloc_n(eng, &dp, nk));
        GF_CU(cudaMemcpy(dp, t.data(), sizeof(EmCls<float>) * nk, cudaMemcpyHostToDevice));
        eng->em_cls_tab = dp;
    } else {
        std::vector<EmCls<double>> t(nk);
        for (size_t c = 0; c < nk; c++) { unsigned ids[4]; ids_of(keys[c], ids); t[c] = em_class<double>(d, ids, P.dt_e0); }
        EmCls<double>* dp = nullptr;
        GF_TRY(dalloc_n(eng, &dp, nk));
        GF_CU(cudaMemcpy(dp, t.data(), sizeof(EmCls<double>) * nk, cudaMemcpyHostToDevice));
        eng->em_cls_tab = dp;
    }
    for (int C = 0; C < 3; C++) {
        GF_TRY(dalloc_n(eng, &eng->ecls[C], cls[C].size()));
        GF_CU(cudaMemcpy(eng->ecls[C], cls[C].data(), cls[C].size(), cudaMemcpyHostToDevice));
    }
    eng->em_ncls = (int)nk;
    P.em_cls = 1;
    return GF_OK;
}

// Set-up from eng->deck (filled from a deck directory or from the host's
// parsed values); `dir` is where restart files are read from ("" = none).
// TMA tensor maps of k_elastic_tile: per step parity and stage, one 3-D map
// (x = k, y = j, z = i) per component of the stage's input displacement and
// one of the material ids, each with the box of one staged plane.  Used only
// when every row stride is a multiple of 16 bytes (nz even in FP64, a
// multiple of 4 in FP32, of 16 for the one-byte ids) and the driver exports
// the encoder; otherwise every block stages with cp.async.
int etile_maps(gf_engine* eng) {
    const Params& P = eng->P;
    if (!eng->tma_err) GF_TRY(dalloc_n(eng, &eng->tma_err, 1));
    for (auto& row : eng->etm)
        for (ETileMaps& m : row) { std::memset(&m, 0, sizeof(m)); m.err = eng->tma_err; m.on = 0; }
    if (!P.elastic) return GF_OK;
    // GOFERRO_TILE_TMA=0 keeps every block on the cp.async staging (the
    // tests check that both stagings give the same bits)
    if (const char* v = std::getenv("GOFERRO_TILE_TMA"))
        if (v[0] == '0') return GF_OK;
    const size_t esz = eng->esz;
    if (P.nz % 16 != 0 || ((size_t)P.nz * esz) % 16 != 0) return GF_OK;
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn) {
        cudaGetLastError();
        return GF_OK;
    }
    auto encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    const cuuint64_t dims[3] = {(cuuint64_t)P.nz, (cuuint64_t)P.ny, (cuuint64_t)P.nx};
    const cuuint32_t estr[3] = {1, 1, 1};
    auto make = [&](CUtensorMap* m, void* base, CUtensorMapDataType t, size_t bytes, cuuint32_t box0) -> bool {
        const cuuint64_t str[2] = {(cuuint64_t)P.nz * bytes, (cuuint64_t)P.ny * P.nz * bytes};
        const cuuint32_t box[3] = {box0, (cuuint32_t)etile::UR, 1};
        return encode(m, t, 3, base, dims, str, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    for (int par = 0; par < 2; par++)
        for (int s = 0; s < 4; s++) {
            ETileMaps& m = eng->etm[par][s];
            bool ok = make(&m.id, eng->mid, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, (cuuint32_t)etile::IP);
            for (int a = 0; a < 3 && ok; a++) {
                if (eng->mixed)
                    ok = make(&m.u[a], (void*)eng->iof[par][s].u_in.c[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                              (cuuint32_t)etile::UP<float>);
                else
                    ok = make(&m.u[a], (void*)eng->io[par][s].u_in.c[a], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8,
                              (cuuint32_t)etile::UP<double>);
            }
            m.on = ok ? 1 : 0;
        }
    return GF_OK;
}

int create_from(gf_engine* eng, const std::string& dir, int device, int precision) {
    if (precision != GF_PRECISION_FP64 && precision != GF_PRECISION_MIXED_FP32) {
        eng->err = "precision must be GF_PRECISION_FP64 or GF_PRECISION_MIXED_FP32";
        return GF_EINVAL;
    }
    eng->mixed = (precision == GF_PRECISION_MIXED_FP32);
    eng->esz = eng->mixed ? sizeof(float) : sizeof(double);
    const Deck& d = eng->deck;
    std::string e = unsupported(d);
    if (!e.empty()) { eng->err = e; return GF_EUNSUPPORTED; }

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { eng->err = "no CUDA device"; return GF_ENODEV; }
    if (device < 0) GF_CU(cudaGetDevice(&device));
    GF_CU(cudaSetDevice(device));
    eng->device = device;
    cudaDeviceProp prop;
    GF_CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) { eng->err = std::string("device ") + prop.name + " is not sm_100 or newer"; return GF_ENODEV; }
    for (cudaEvent_t& ev : eng->bev) GF_CU(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));

    build_params(eng);
    const Params& P = eng->P;
    {
        // Priorities of the stage kernels' streams, kept by the step
        // graph's kernel nodes (cudaGraphInstantiateFlagUseNodePriority).
        // Without magnets the elastic chain of the engine stream (tile, RK
        // update) is the longest of a stage and goes first, then the
        // Maxwell update and the TDGL kernel in the order measured faster
        // for each form (128^3 ferroelectric, ms per step: FP64 2.453 ->
        // 2.357 with Maxwell before TDGL, which waits for the tile there;
        // FP32 1.422 -> 1.354 with TDGL before Maxwell).  With magnets the
        // LLG and Maxwell kernels wait for the tile and RK update is off the
        // critical path: equal priorities (128x128x96 magnetoelastic: the
        // elastic-first order measured 0.878 -> 0.905 ms FP32, 1.491 ->
        // 1.521 FP64; branches first 0.880 / 1.492).
        int lo = 0, hi = 0;
        GF_CU(cudaDeviceGetStreamPriorityRange(&lo, &hi));
        const int mid = (lo + hi) / 2;
        int pm = lo, pl = lo, pf = lo, pe = lo;
        if (P.elastic && !(P.fm || P.afm)) {
            pm = hi;
            if (eng->mixed) pf = mid; else pe = mid;
        }
        eng->prio_nodes = pm != lo || pf != lo || pe != lo;
        GF_CU(cudaStreamCreateWithPriority(&eng->stream, cudaStreamNonBlocking, pm));
        GF_CU(cudaStreamCreateWithPriority(&eng->side[0], cudaStreamNonBlocking, pl));
        GF_CU(cudaStreamCreateWithPriority(&eng->side[1], cudaStreamNonBlocking, pf));
        GF_CU(cudaStreamCreateWithPriority(&eng->side[2], cudaStreamNonBlocking, pe));
    }
    const long n = P.n;
    if (eng->mixed) {
        e = unsupported_mixed(d, P);
        if (!e.empty()) { eng->err = e; return GF_EUNSUPPORTED; }
    }

    // materials
    GF_TRY(dalloc_n(eng, &eng->mid, (size_t)n));
    GF_CU(cudaMemcpyAsync(eng->mid, d.material_cell.data(), (size_t)n, cudaMemcpyHostToDevice, eng->stream));
    std::vector<DevMat> dm(d.mats.size());
    for (size_t i = 0; i < d.mats.size(); i++) dm[i] = make_devmat(d.mats[i], d.dt);
    GF_TRY(dalloc_n(eng, &eng->mats, dm.size()));
    GF_CU(cudaMemcpyAsync(eng->mats, dm.data(), sizeof(DevMat) * dm.size(), cudaMemcpyHostToDevice, eng->stream));
    if (eng->mixed) {
        std::vector<DevMatT<float>> dmf(dm.size());
        for (size_t i = 0; i < dm.size(); i++) dmf[i] = devmat_f32(dm[i]);
        GF_TRY(dalloc_n(eng, &eng->mats_f, dmf.size()));
        GF_CU(cudaMemcpy(eng->mats_f, dmf.data(), sizeof(DevMatT<float>) * dmf.size(), cudaMemcpyHostToDevice));
    }
    {
        LLGTables t;
        std::memset(&t, 0, sizeof(t));
        for (size_t a = 0; a < d.mats.size(); a++)
            for (size_t b = 0; b < d.mats.size(); b++) {
                const double A1 = d.mats[a].Aex, A2 = d.mats[b].Aex;
                t.Aij[a + 1][b + 1] = (A1 + A2 != 0.) ? 2. * A1 * A2 / (A1 + A2) : 0.;
                // magnetic_initialize.cpp:877-1071: 2 A1 A2 / (A1 + A2) per sublattice
                const double B1[2] = {d.mats[a].Aex1, d.mats[a].Aex2}, B2[2] = {d.mats[b].Aex1, d.mats[b].Aex2};
                for (int s = 0; s < 2; s++)
                    t.AijA[s][a + 1][b + 1] = (B1[s] + B2[s] != 0.) ? 2. * B1[s] * B2[s] / (B1[s] + B2[s]) : 0.;
            }
        GF_TRY(dalloc_n(eng, &eng->llg_tab, 1));
        GF_CU(cudaMemcpy(eng->llg_tab, &t, sizeof(t), cudaMemcpyHostToDevice));
        if (eng->mixed) {
            LLGTablesT<float> tf;
            for (int a = 0; a <= kMaxMat; a++)
                for (int b = 0; b <= kMaxMat; b++) {
                    tf.Aij[a][b] = (float)t.Aij[a][b];
                    for (int s = 0; s < 2; s++) tf.AijA[s][a][b] = (float)t.AijA[s][a][b];
                }
            GF_TRY(dalloc_n(eng, &eng->llg_tab_f, 1));
            GF_CU(cudaMemcpy(eng->llg_tab_f, &tf, sizeof(tf), cudaMemcpyHostToDevice));
        }
    }
    GF_TRY(dalloc_n(eng, &eng->drive, (size_t)kDriveCap));
    GF_CU(cudaMallocHost(&eng->drive_host, sizeof(StepDrive) * kDriveCap));
    GF_TRY(dalloc_n(eng, &eng->step_ctr, 1));
    {
        std::vector<double> kf((size_t)P.nz, 0.);
        if (d.jf_input) {
            const double PI = kPi;
            const long Jf_nz = (long)(d.jf_k1 - d.jf_k0 + 1);
            for (long k = (long)d.jf_k0; k <= (long)d.jf_k1 && k < P.nz; k++) {
                const double sp = PI / (static_cast<double>(Jf_nz) * P.dz) * (static_cast<double>(k - (long)d.jf_k0) + 0.5) * P.dz;
                kf[(size_t)k] = (d.jf_type == 1) ? std::sin(sp) : std::cos(sp);
            }
        }
        GF_TRY(dalloc_r(eng, &eng->jf_kfac, (size_t)P.nz));
        GF_TRY(upload_one(eng, eng->jf_kfac, nullptr, kf.data(), (long)kf.size()));
    }

    // spin pumping layers (global.cpp:168-240) and the per-k coefficient of
    // get_J_ISHE_RK* (magnetic_solver.cpp:241-261): coeff_Js * coeff_L
    if (P.spin) {
        const double PI = kPi, unit_e = 1.602176634e-19;    // magnetic_system.h:15-16
        std::vector<int> src((size_t)P.nz, -1);
        std::vector<double> thick((size_t)P.nz, 0.), coef((size_t)P.nz, 0.);
        auto mat_at_k = [&](long k) -> unsigned { return d.material_cell[(size_t)k]; };   // cell (0,0,k)
        auto magnetic = [&](unsigned id) { return id != 0 && (d.mats[id - 1].fm || d.mats[id - 1].afm); };
        long id_zf = (long)d.idzi - 1;
        for (size_t L = 0; L < d.nz_layer.size(); L++) {
            const long id_zi = id_zf + 1;
            id_zf = id_zi + (long)d.nz_layer[L] - 1;
            const unsigned mt = mat_at_k(id_zi);
            if (mt == 0 || !d.mats[mt - 1].spin_pump) continue;
            const bool si = id_zi != 0 && magnetic(mat_at_k(id_zi - 1));
            const bool sf = id_zf != P.nz - 1 && magnetic(mat_at_k(id_zf + 1));
            long s = -1;
            if (si && !sf) s = id_zi - 1;
            else if (!si && sf) s = id_zf + 1;
            if (s < 0) continue;
            for (long k = id_zi; k <= id_zf && k < P.nz; k++) { src[(size_t)k] = (int)s; thick[(size_t)k] = d.nz_layer[L] * P.dz; }
        }
        for (long k = 0; k < P.nz; k++) {
            if (src[(size_t)k] < 0) continue;
            const Material& m = d.mats[mat_at_k(k) - 1];
            const double coeff_Js = m.sh_angle * unit_e / 2. / PI * m.sh_mixcond;
            const double distance = (std::abs(static_cast<double>((k - src[(size_t)k]))) - 0.5) * P.dz;
            double coeff_L;
            if (k > src[(size_t)k])
                coeff_L = std::sinh((thick[(size_t)k] - distance) / m.sh_difflen) / std::sinh(thick[(size_t)k] / m.sh_difflen);
            else
                coeff_L = -1. * std::sinh((thick[(size_t)k] - distance) / m.sh_difflen) / std::sinh(thick[(size_t)k] / m.sh_difflen);
            coef[(size_t)k] = coeff_Js * coeff_L;
        }
        GF_TRY(dalloc_r(eng, &eng->ishe_coef, (size_t)P.nz));
        GF_TRY(dalloc_n(eng, &eng->ishe_src, (size_t)P.nz));
        GF_CU(cudaStreamSynchronize(eng->stream));
        GF_TRY(upload_one(eng, eng->ishe_coef, nullptr, coef.data(), P.nz));
        GF_CU(cudaMemcpy(eng->ishe_src, src.data(), sizeof(int) * P.nz, cudaMemcpyHostToDevice));
    }

    // state fields
    if (d.any_fm) GF_TRY(alloc_field(eng, eng->m, n, n, n));
    if (d.any_afm) { GF_TRY(alloc_field(eng, eng->a1, n, n, n)); GF_TRY(alloc_field(eng, eng->a2, n, n, n)); }
    if (P.drude)
        for (int pole = 0; pole < 3; pole++) GF_TRY(alloc_field(eng, eng->jp[pole], n, n, n));
    if (d.any_fe) { GF_TRY(alloc_field(eng, eng->p, n, n, n)); GF_TRY(alloc_field(eng, eng->q, n, n, n)); }
    if (d.elastodynamics) { GF_TRY(alloc_field(eng, eng->u, n, n, n)); GF_TRY(alloc_field(eng, eng->v, n, n, n)); }
    if (d.em_dynamic) {
        const long nx = P.nx, ny = P.ny, nz = P.nz;
        GF_TRY(alloc_field(eng, eng->E, nx * (ny + 1) * (nz + 1), (nx + 1) * ny * (nz + 1), (nx + 1) * (ny + 1) * nz));
        GF_TRY(alloc_field(eng, eng->H, (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)));
    }
    for (int a = 0; a < 3; a++) {
        if (P.em_fromM || P.spin) GF_TRY(dalloc_r(eng, &eng->dm[a], (size_t)n));
        if ((P.em_fromM || P.spin) && d.any_afm) { GF_TRY(dalloc_r(eng, &eng->da1[a], (size_t)n)); GF_TRY(dalloc_r(eng, &eng->da2[a], (size_t)n)); }
        if (d.elastodynamics) {
            GF_TRY(dalloc_r(eng, &eng->force_store[a], (size_t)n));
            GF_TRY(dalloc_r(eng, &eng->force[a], (size_t)n));
        }
        // with the FFT magnetostatics H_stat is a view of the FFT buffer (setup_demag)
        if ((d.any_fm || d.any_afm) && !(d.magnetostatics && !d.mag_1D && !d.demag_factor))
            GF_TRY(dalloc_r(eng, &eng->Hstat[a], (size_t)n));
        if (d.any_fe) GF_TRY(dalloc_r(eng, &eng->Estat[a], (size_t)n));
        if (d.any_fm && d.read_Hext_nonunif) GF_TRY(dalloc_r(eng, &eng->Hnu[a], (size_t)n));
    }
    if (d.elastodynamics)
        for (int a = 0; a < 9; a++) GF_TRY(dalloc_r(eng, &eng->fg[a], (size_t)n));
    // the crystal-frame cell strain the elastic tile hands to the LLG kernels
    // and to the FP64 TDGL kernel
    if (d.elastodynamics && P.elasto_on && (P.fm || P.afm || (P.fe && !eng->mixed)))
        for (int a = 0; a < 6; a++) GF_TRY(dalloc_r(eng, &eng->strain_c[a], (size_t)n));
    // flexoelectricity: global-frame cell strain and eigenstrain p-gradients
    // of the stage state (k_flexo_prep)
    if (P.flexo)
        for (int a = 0; a < 6; a++) {
            if (d.elastodynamics) GF_TRY(dalloc_r(eng, &eng->flexo_sg[a], (size_t)n));
            GF_TRY(dalloc_r(eng, &eng->flexo_pge[a], (size_t)n));
        }
    if (d.elastodynamics) GF_TRY(setup_elastic_tile(eng));
    if (d.elastodynamics) {
        const size_t plane = (size_t)P.nx * P.ny;
        GF_TRY(dalloc_r(eng, &eng->liao_hist, 4 * 12 * plane));
        GF_TRY(dalloc_r(eng, &eng->liao_last, 3 * plane));
    }
    if (P.em) GF_TRY(setup_em_classes(eng));
    // FP64 scratch: output staging (6 cell arrays, or one widened Yee
    // component in the mixed form) and the reduction partials (device_sum3:
    // 3 x (592 + 1); the adjoint's means: 8192 + 64 + 1)
    const size_t yee_max = (size_t)(P.nx + 1) * (P.ny + 1) * (P.nz + 1);
    eng->scratch_main = std::max((size_t)6 * n, yee_max);
    GF_TRY(dalloc_n(eng, &eng->scratch, eng->scratch_main + 32768));
    GF_TRY(dalloc_n(eng, &eng->flag, 1));
    GF_CU(cudaStreamSynchronize(eng->stream));

    GF_TRY(setup_demag(eng));          // before the restart inputs: Hstat.in lands in the FFT buffer
    GF_TRY(initial_state(eng, dir));
    GF_TRY(replicate_state(eng));
    build_io(eng);
    if (eng->mixed) build_io_mixed(eng);
    GF_TRY(etile_maps(eng));

    // initial static field (main.cpp:135-146 and 229-239)
    if (!d.in_Hstat) GF_TRY(static_field_now(eng));
    GF_CU(cudaStreamSynchronize(eng->stream));
    return GF_OK;
}

int create(gf_engine* eng, const std::string& dir, int device, int precision) {
    std::string e = read_deck(dir, eng->deck);
    if (!e.empty()) { eng->err = e; return GF_EIO; }
    return create_from(eng, dir, device, precision);
}

// the captured step graphs hold Params by value: drop them after a change
void invalidate_graphs(gf_engine* eng) {
    eng->graphs_ready = false;
    for (int p = 0; p < 2; p++) {
        if (eng->gexec[p]) { cudaGraphExecDestroy(eng->gexec[p]); eng->gexec[p] = nullptr; }
        if (eng->graph[p]) { cudaGraphDestroy(eng->graph[p]); eng->graph[p] = nullptr; }
    }
}

// E_stat stops being known to be +0 everywhere (the TDGL kernel then reads it)
void mark_estat(gf_engine* eng) {
    if (eng->P.estat || !eng->Estat[0]) return;
    eng->P.estat = 1;
    invalidate_graphs(eng);
}

int ensure_graphs(gf_engine* eng) {
    if (eng->graphs_ready) return GF_OK;
    for (int par = 0; par < 2; par++) {
        GF_CU(cudaStreamBeginCapture(eng->stream, cudaStreamCaptureModeThreadLocal));
        int rc = enqueue_step(eng, par);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(eng->stream, &g);
        if (rc != GF_OK) { if (g) cudaGraphDestroy(g); return rc; }
        if (ce != cudaSuccess) { eng->err = std::string("stream capture: ") + cudaGetErrorString(ce); return GF_ECUDA; }
        eng->graph[par] = g;
        GF_CU(cudaGraphInstantiate(&eng->gexec[par], g, eng->prio_nodes ? cudaGraphInstantiateFlagUseNodePriority : 0));
    }
    eng->graphs_ready = true;
    return GF_OK;
}

int advance(gf_engine* eng, uint64_t nsteps, bool use_graph) {
    if (eng->stage_open) {
        eng->err = "a step begun with gf_stage_begin is still open (commit its stages first)";
        return GF_EINVAL;
    }
    if (use_graph) GF_TRY(ensure_graphs(eng));
    eng->stage_done = 0;
    uint64_t done = 0;
    while (done < nsteps) {
        const uint64_t chunk = std::min<uint64_t>(nsteps - done, (uint64_t)kDriveCap / 2);
        // the device drive ring holds kDriveCap steps; steps are written at
        // slot (step & (kDriveCap-1)); wait for earlier users of the pinned buffer
        GF_CU(cudaStreamSynchronize(eng->stream));
        for (uint64_t s = 0; s < chunk; s++) step_drive(eng, eng->drive_host[s]);
        const uint64_t first = eng->steps_done + done;
        uint64_t s = 0;
        while (s < chunk) {
            const uint64_t slot = (first + s) & (uint64_t)(kDriveCap - 1);
            const uint64_t run = std::min<uint64_t>(chunk - s, (uint64_t)kDriveCap - slot);
            GF_CU(cudaMemcpyAsync(eng->drive + slot, eng->drive_host + s, sizeof(StepDrive) * run, cudaMemcpyHostToDevice, eng->stream));
            s += run;
        }
        for (uint64_t k = 0; k < chunk; k++) {
            const int parity = (int)((first + k) & 1ull);
            if (use_graph) GF_CU(cudaGraphLaunch(eng->gexec[parity], eng->stream));
            else GF_TRY(enqueue_step(eng, parity));
        }
        done += chunk;
    }
    eng->steps_done += nsteps;
    return GF_OK;
}

// current step value of a 3-component state field
double* const* cur(gf_engine* eng, Field3& f) { return (eng->steps_done & 1ull) ? f.A : f.X; }

// Deterministic FP64 sums of three device arrays of the run's precision (in
// the mixed form of the values x + c when the compensation words c are
// given): 8192 strided partials, then 64, then 1, each sum in a fixed order;
// one copy back and one synchronisation for the three
// gf_average's reductions: one pass into kSumBlocks partials per component
// (warp-shuffle block sums), one pass over the partials, one read-back
constexpr int kSumBlocks = 592;
int device_sum3(gf_engine* eng, double* const* in, long n, double out[3], double* const* cmp) {
    cudaStream_t st = eng->stream;
    double* p1 = eng->scratch + eng->scratch_main;            // 3 x kSumBlocks
    double* p3 = p1 + 3 * kSumBlocks;                         // 3
    Sum3In a{};
    a.f32 = eng->mixed ? 1 : 0;
    for (int c = 0; c < 3; c++) { a.x[c] = in[c]; a.cm[c] = eng->mixed && cmp ? reinterpret_cast<const float*>(cmp[c]) : nullptr; }
    GF_CU(launch(k_sum3_block, dim3(kSumBlocks, 3), dim3(kSumThreads), 0, st, a, n, p1));
    GF_CU(launch(k_sum3_final, dim3(3), dim3(kSumThreads), 0, st, (const double*)p1, kSumBlocks, p3));
    GF_CU(cudaMemcpyAsync(out, p3, 3 * sizeof(double), cudaMemcpyDeviceToHost, st));
    GF_CU(cudaStreamSynchronize(st));
    return GF_OK;
}

// cell-centred E and H (scratch[0..3n) and scratch[3n..6n)) of cells c0 ..
// c0 + count - 1 of the current step value
int em_cells(gf_engine* eng, long c0, long count) {
    const Params& P = eng->P;
    double* s = eng->scratch;
    F3 Ec{{s, s + P.n, s + 2 * P.n}}, Hc{{s + 3 * P.n, s + 4 * P.n, s + 5 * P.n}};
    if (eng->mixed)
        GF_CU(launch(k_em_cell<float>, dim3(blocks_for(count, kThreads)), dim3(kThreads), 0, eng->stream, P,
                     f3f(cur(eng, eng->E)), f3f(cur(eng, eng->H)), Ec, Hc, c0, count));
    else
        GF_CU(launch(k_em_cell<double>, dim3(blocks_for(count, kThreads)), dim3(kThreads), 0, eng->stream, P,
                     f3(cur(eng, eng->E)), f3(cur(eng, eng->H)), Ec, Hc, c0, count));
    if (P.mag1d_em) {
        // H_z of the 1-D model in place of the face mean
        const double* mz = (eng->deck.any_fm) ? cur(eng, eng->m)[2] : nullptr;
        const double* z1 = (eng->deck.any_afm) ? cur(eng, eng->a1)[2] : nullptr;
        const double* z2 = (eng->deck.any_afm) ? cur(eng, eng->a2)[2] : nullptr;
        if (eng->mixed)
            GF_CU(launch(k_em_cell_hz_1d<float>, dim3(blocks_for(count, kThreads)), dim3(kThreads), 0, eng->stream,
                         (const DevMatT<float>*)eng->mats_f, (const uint8_t*)eng->mid, (const float*)mz, (const float*)z1,
                         (const float*)z2, (const float*)eng->Hstat[2], Hc.c[2], c0, count));
        else
            GF_CU(launch(k_em_cell_hz_1d<double>, dim3(blocks_for(count, kThreads)), dim3(kThreads), 0, eng->stream,
                         (const DevMatT<double>*)eng->mats, (const uint8_t*)eng->mid, mz, z1, z2, (const double*)eng->Hstat[2],
                         Hc.c[2], c0, count));
    }
    return GF_OK;
}

// Device arrays of a field, component by component.  `native` is true when
// they are state buffers of the run's precision (FP32 in the mixed form, with
// compensation words in `cmps`, null where the field has none) and false
// when they are FP64 output staged in the scratch buffer.
int field_ptrs(gf_engine* eng, int field, std::vector<double*>& ptrs, std::vector<long>& lens, bool& writable,
               std::vector<double*>& cmps, bool& native) {
    const Params& P = eng->P;
    writable = true;
    native = true;
    ptrs.clear(); lens.clear(); cmps.clear();
    auto add3 = [&](double* const* p, Field3* f) {
        for (int a = 0; a < 3; a++) {
            ptrs.push_back(p[a]);
            lens.push_back(f ? f->len[a] : P.n);
            cmps.push_back(f ? f->C[a] : nullptr);
        }
    };
    switch (field) {
        case GF_FIELD_M: if (!eng->m.on) break; add3(cur(eng, eng->m), &eng->m); break;
        case GF_FIELD_M_AFM1: if (!eng->a1.on) break; add3(cur(eng, eng->a1), &eng->a1); break;
        case GF_FIELD_M_AFM2: if (!eng->a2.on) break; add3(cur(eng, eng->a2), &eng->a2); break;
        case GF_FIELD_P: if (!eng->p.on) break; add3(cur(eng, eng->p), &eng->p); break;
        case GF_FIELD_Q: if (!eng->q.on) break; add3(cur(eng, eng->q), &eng->q); break;
        case GF_FIELD_U: if (!eng->u.on) break; add3(cur(eng, eng->u), &eng->u); break;
        case GF_FIELD_V: if (!eng->v.on) break; add3(cur(eng, eng->v), &eng->v); break;
        case GF_FIELD_EX: case GF_FIELD_EY: case GF_FIELD_EZ: {
            if (!eng->E.on) break;
            const int a = field - GF_FIELD_EX;
            ptrs.push_back(cur(eng, eng->E)[a]); lens.push_back(eng->E.len[a]); cmps.push_back(eng->E.C[a]); break;
        }
        case GF_FIELD_HX: case GF_FIELD_HY: case GF_FIELD_HZ: {
            if (!eng->H.on) break;
            const int a = field - GF_FIELD_HX;
            ptrs.push_back(cur(eng, eng->H)[a]); lens.push_back(eng->H.len[a]); cmps.push_back(eng->H.C[a]); break;
        }
        case GF_FIELD_HSTAT: if (!eng->Hstat[0]) break; add3(eng->Hstat, nullptr); break;
        case GF_FIELD_STRAIN_STATIC: case GF_FIELD_EIGENSTRAIN_STATIC: {
            double* const* f = (field == GF_FIELD_STRAIN_STATIC) ? eng->es_eps : eng->es_eig;
            if (!f[0]) break;
            for (int a = 0; a < 6; a++) { ptrs.push_back(f[a]); lens.push_back(P.n); cmps.push_back(nullptr); }
            break;
        }
        case GF_FIELD_ESTAT: if (!eng->Estat[0]) break; add3(eng->Estat, nullptr); break;
        case GF_FIELD_FORCE_STORE: if (!eng->force_store[0]) break; add3(eng->force_store, nullptr); break;
        case GF_FIELD_JP1: case GF_FIELD_JP2: case GF_FIELD_JP3: {
            Field3& f = eng->jp[field - GF_FIELD_JP1];
            if (!f.on) break;
            add3(cur(eng, f), &f);
            break;
        }
        case GF_FIELD_E_CELL: case GF_FIELD_H_CELL: {
            if (!eng->E.on) break;
            writable = false;
            native = false;
            double* s = eng->scratch;
            GF_TRY(em_cells(eng, 0, P.n));
            double* base = (field == GF_FIELD_E_CELL) ? s : s + 3 * P.n;
            for (int a = 0; a < 3; a++) { ptrs.push_back(base + a * P.n); lens.push_back(P.n); cmps.push_back(nullptr); }
            break;
        }
        case GF_FIELD_STRAIN: {
            // strain of the current step value (face gradients recomputed from it)
            if (!eng->u.on) break;
            writable = false;
            native = false;
            const int par = (int)(eng->steps_done & 1ull);
            if (eng->mixed) {
                StageIOT<float> io = eng->iof[par][0];
                GF_CU(launch(k_face_grad<float>, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, eng->stream, P, io));
                GF_CU(launch(k_cell_strain<float>, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, eng->stream, P, io, eng->scratch));
            } else {
                StageIO io = eng->io[par][0];
                GF_CU(launch(k_face_grad<double>, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, eng->stream, P, io));
                GF_CU(launch(k_cell_strain<double>, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, eng->stream, P, io, eng->scratch));
            }
            for (int a = 0; a < 6; a++) { ptrs.push_back(eng->scratch + (size_t)a * P.n); lens.push_back(P.n); cmps.push_back(nullptr); }
            break;
        }
        default: break;
    }
    if (ptrs.empty()) { eng->err = "field " + std::to_string(field) + " is not present in this run"; return GF_EINVAL; }
    return GF_OK;
}

int check(gf_engine* e) {
    if (!e) return GF_EINVAL;
    return GF_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
namespace {

// the 1-D electrostatic field of the current polarisation (state `parity`)
int elec_1d_now(gf_engine* eng, int parity) {
    const Params& P = eng->P;
    const dim3 g(blocks_for((long)P.nx * P.ny, kThreads));
    if (eng->mixed) {
        const StageIOT<float>& io = eng->iof[parity][0];
        GF_CU(launch(k_elec_1d<float>, g, dim3(kThreads), 0, eng->stream, P, io.mats, io.mid, (const float*)io.p_in.c[2],
                     (const float*)reinterpret_cast<float*>(eng->elec_pz_t0), io.Estat));
    } else {
        const StageIO& io = eng->io[parity][0];
        GF_CU(launch(k_elec_1d<double>, g, dim3(kThreads), 0, eng->stream, P, io.mats, io.mid, (const double*)io.p_in.c[2],
                     (const double*)eng->elec_pz_t0, io.Estat));
    }
    return GF_OK;
}

// One elastostatic solve from the state of `parity` (its stage-1 inputs):
// the static eigenstrain, then up to `iters` Khachaturyan iterations from the
// last solution (gf_elasto.cuh), stopping early at `tol` when tol > 0 (host
// checks, not inside a capture); the result goes to the static strain arrays
int es_solve(gf_engine* eng, int parity, bool counted, int iters, double tol, int* used) {
    const Params& P = eng->P;
    cudaStream_t st = eng->stream;
    const long n = P.n, n21 = (long)P.nx * P.ny * (P.nz / 2 + 1);
    const unsigned bn = blocks_for(n, kThreads);
    auto L = [&](const char* name, auto k, dim3 g, dim3 b, auto... args) -> cudaError_t {
        return counted ? klaunch(eng, name, k, g, b, 0, st, args...) : launch(k, g, b, 0, st, args...);
    };
    if (eng->mixed) GF_CU(L("k_es_eigen", k_es_eigen<float>, dim3(bn), dim3(kThreads), P, eng->iof[parity][0], eng->es_e0));
    else GF_CU(L("k_es_eigen", k_es_eigen<double>, dim3(bn), dim3(kThreads), P, eng->io[parity][0], eng->es_e0));
    std::vector<double> bm(2 * kElecBlocks);
    int it = 0;
    for (; it < iters; it++) {
        GF_CU(L("k_es_tau", k_es_tau, dim3(bn), dim3(kThreads), P, (const uint8_t*)eng->mid, eng->es_mats, eng->es_ch[0],
                eng->es_ch[1], eng->es_ch[2], (const double*)eng->es_x, (const double*)eng->es_e0, eng->es_r));
        GF_FFT(cufftExecD2Z(eng->es_r2c, eng->es_r, eng->es_k));
        GF_CU(L("k_es_green", k_es_green, dim3(blocks_for(n21, kThreads)), dim3(kThreads), n21, 1. / (double)n,
                (const double*)eng->es_G, (const double*)eng->es_kq, (const int*)eng->es_nyq_idx,
                (const double*)eng->es_nyq_op, eng->es_k));
        GF_FFT(cufftExecZ2D(eng->es_c2r, eng->es_k, eng->es_r));
        GF_CU(L("k_es_update", k_es_update, dim3(kElecBlocks), dim3(256), n, (const double*)eng->es_r, eng->es_x,
                tol > 0. ? eng->es_blockmax : (double*)nullptr));
        if (tol > 0.) {
            GF_CU(cudaMemcpyAsync(bm.data(), eng->es_blockmax, sizeof(double) * bm.size(), cudaMemcpyDeviceToHost, st));
            GF_CU(cudaStreamSynchronize(st));
            double md = 0., me = 0.;
            for (int b = 0; b < kElecBlocks; b++) { md = std::max(md, bm[2 * b]); me = std::max(me, bm[2 * b + 1]); }
            if (md <= tol * me) { it++; break; }
        }
    }
    if (used) *used = it;
    double* const* o = eng->es_eps;
    double* const* g = eng->es_eig;
    if (eng->mixed) {
        auto f = [](double* x) { return reinterpret_cast<float*>(x); };
        GF_CU(L("k_es_out", k_es_out<float>, dim3(bn), dim3(kThreads), n, (const uint8_t*)eng->mid, (const double*)eng->es_x,
                (const double*)eng->es_e0, f(o[0]), f(o[1]), f(o[2]), f(o[3]), f(o[4]), f(o[5]), f(g[0]), f(g[1]), f(g[2]),
                f(g[3]), f(g[4]), f(g[5])));
    } else {
        GF_CU(L("k_es_out", k_es_out<double>, dim3(bn), dim3(kThreads), n, (const uint8_t*)eng->mid, (const double*)eng->es_x,
                (const double*)eng->es_e0, o[0], o[1], o[2], o[3], o[4], o[5], g[0], g[1], g[2], g[3], g[4], g[5]));
    }
    return GF_OK;
}

// Solver buffers, plans and tables (once per engine): C_h and the crystal-
// frame constants, the wave vectors of global.cpp:276-316 rotated to the
// crystal frame, and the Green tensor of elastic_initialize.cpp:340-389
int es_setup(gf_engine* eng) {
    const Deck& d = eng->deck;
    const Params& P = eng->P;
    const long n = P.n, nz21 = P.nz / 2 + 1, n21 = (long)P.nx * P.ny * nz21;
    // C_h: the largest c11, c12, c44 of all materials, times scale_elasto
    double ch[3] = {d.mats[0].c11, d.mats[0].c12, d.mats[0].c44};
    for (const Material& m : d.mats) { ch[0] = std::max(ch[0], m.c11); ch[1] = std::max(ch[1], m.c12); ch[2] = std::max(ch[2], m.c44); }
    const double scale = d.scale_elasto > 0. ? d.scale_elasto : 1.;
    for (double& c : ch) c = c * scale;
    for (int a = 0; a < 3; a++) eng->es_ch[a] = ch[a];
    std::memset(&eng->es_mats, 0, sizeof(eng->es_mats));
    for (size_t i = 0; i < d.mats.size(); i++) {
        eng->es_mats.c[i + 1][0] = d.mats[i].c11; eng->es_mats.c[i + 1][1] = d.mats[i].c12; eng->es_mats.c[i + 1][2] = d.mats[i].c44;
    }
    if (eng->es_x) return GF_OK;
    if (ch[2] <= 0.) { eng->err = "elastostatics needs a material with c44 > 0"; return GF_EINVAL; }
    const double PI = kPi;
    const long dims[3] = {P.nx, P.ny, P.nz};
    const double h[3] = {P.dx, P.dy, P.dz};
    std::vector<double> kv[3];
    for (int a = 0; a < 3; a++) {
        const long len = (a < 2) ? dims[a] : nz21;
        kv[a].resize((size_t)len);
        const double dk = 2. * PI / (static_cast<double>(dims[a]) * h[a]);
        for (long i = 0; i < len; i++) {
            long t = i;
            if (t > dims[a] / 2) t = t - dims[a];
            kv[a][(size_t)i] = static_cast<double>(t) * dk;
        }
    }
    const double c11 = ch[0], c12 = ch[1], c44 = ch[2];
    const double chi = (c11 - c12 - 2. * c44) / c44;
    // crystal-frame wave vector and Green tensor of one global wave vector
    auto green = [&](double kx, double ky, double kz, double kq[3], double g[6]) {
        double a = kx, b = ky, c = kz;
        if (d.orient_rotate) {
            a = d.Tg2c[0][0] * kx + d.Tg2c[0][1] * ky + d.Tg2c[0][2] * kz;
            b = d.Tg2c[1][0] * kx + d.Tg2c[1][1] * ky + d.Tg2c[1][2] * kz;
            c = d.Tg2c[2][0] * kx + d.Tg2c[2][1] * ky + d.Tg2c[2][2] * kz;
        }
        const double kn = std::pow(kz, 2.) + std::pow(ky, 2.) + std::pow(kx, 2.);
        const double a2 = a * a, b2 = b * b, c2 = c * c;
        const double d0 = (kn < 1.e-8) ? 1.
            : c11 * std::pow(kn, 3.) + chi * (c11 + c12) * kn * (a2 * b2 + b2 * c2 + c2 * a2)
              + chi * chi * (c11 + 2 * c12 + c44) * a2 * b2 * c2;
        const double den = c44 * d0;
        g[0] = (c44 * std::pow(kn, 2.) + (c11 + c12) * chi * b2 * c2 + (c11 - c44) * kn * (b2 + c2)) / den;
        g[1] = (c44 * std::pow(kn, 2.) + (c11 + c12) * chi * c2 * a2 + (c11 - c44) * kn * (c2 + a2)) / den;
        g[2] = (c44 * std::pow(kn, 2.) + (c11 + c12) * chi * a2 * b2 + (c11 - c44) * kn * (a2 + b2)) / den;
        g[3] = -(c12 + c44) * (kn + chi * c2) * a * b / den;
        g[4] = -(c12 + c44) * (kn + chi * b2) * a * c / den;
        g[5] = -(c12 + c44) * (kn + chi * a2) * b * c / den;
        kq[0] = a; kq[1] = b; kq[2] = c;
    };
    // the 6 x 6 operator tau (Voigt order, tensor components) -> de of one
    // wave vector, accumulated into M with weight w
    auto op6 = [&](double kx, double ky, double kz, double w, double* M) {
        double kq[3], g[6];
        green(kx, ky, kz, kq, g);
        const double Gm[3][3] = {{g[0], g[3], g[4]}, {g[3], g[1], g[5]}, {g[4], g[5], g[2]}};
        const int pi_[6] = {0, 1, 2, 1, 0, 0}, pj[6] = {0, 1, 2, 2, 2, 1};
        for (int bcol = 0; bcol < 6; bcol++) {
            double t[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            t[pi_[bcol]][pj[bcol]] = 1.; t[pj[bcol]][pi_[bcol]] = 1.;
            double f[3], nv[3];
            for (int i = 0; i < 3; i++) f[i] = t[i][0] * kq[0] + t[i][1] * kq[1] + t[i][2] * kq[2];
            for (int i = 0; i < 3; i++) nv[i] = Gm[i][0] * f[0] + Gm[i][1] * f[1] + Gm[i][2] * f[2];
            for (int arow = 0; arow < 6; arow++) {
                const int i = pi_[arow], j = pj[arow];
                M[6 * arow + bcol] += w * 0.5 * (kq[j] * nv[i] + kq[i] * nv[j]);
            }
        }
    };
    std::vector<double> G((size_t)6 * n21), KQ((size_t)3 * n21), NOP;
    std::vector<int> NIDX((size_t)n21, -1);
    for (long i = 0; i < P.nx; i++)
        for (long j = 0; j < P.ny; j++)
            for (long k = 0; k < nz21; k++) {
                const long q = (i * P.ny + j) * nz21 + k;
                const double kx = kv[0][(size_t)i], ky = kv[1][(size_t)j], kz = kv[2][(size_t)k];
                double kq[3], g[6];
                green(kx, ky, kz, kq, g);
                for (int a = 0; a < 6; a++) G[(size_t)(a * n21 + q)] = g[a];
                for (int a = 0; a < 3; a++) KQ[(size_t)(a * n21 + q)] = kq[a];
                const bool nyq[3] = {P.nx % 2 == 0 && i == P.nx / 2, P.ny % 2 == 0 && j == P.ny / 2,
                                     P.nz % 2 == 0 && k == P.nz / 2};
                if (!(nyq[0] || nyq[1] || nyq[2])) continue;
                const int m = (int)nyq[0] + (int)nyq[1] + (int)nyq[2];
                NIDX[(size_t)q] = (int)(NOP.size() / 36);
                NOP.resize(NOP.size() + 36, 0.);
                double* M = NOP.data() + NOP.size() - 36;
                for (int sgn = 0; sgn < 8; sgn++) {
                    // flip only the Nyquist components; 2^m distinct combinations
                    if (((sgn & 1) && !nyq[0]) || ((sgn & 2) && !nyq[1]) || ((sgn & 4) && !nyq[2])) continue;
                    op6((sgn & 1) ? -kx : kx, (sgn & 2) ? -ky : ky, (sgn & 4) ? -kz : kz, 1. / (double)(1 << m), M);
                }
            }
    GF_TRY(dalloc_n(eng, &eng->es_x, (size_t)6 * n));
    GF_TRY(dalloc_n(eng, &eng->es_e0, (size_t)6 * n));
    GF_TRY(dalloc_n(eng, &eng->es_r, (size_t)6 * n));
    GF_TRY(dalloc_n(eng, &eng->es_k, (size_t)6 * n21));
    GF_TRY(dalloc_n(eng, &eng->es_G, (size_t)6 * n21));
    GF_TRY(dalloc_n(eng, &eng->es_kq, (size_t)3 * n21));
    GF_TRY(dalloc_n(eng, &eng->es_blockmax, (size_t)2 * kElecBlocks));
    GF_CU(cudaMemcpy(eng->es_G, G.data(), sizeof(double) * G.size(), cudaMemcpyHostToDevice));
    GF_CU(cudaMemcpy(eng->es_kq, KQ.data(), sizeof(double) * KQ.size(), cudaMemcpyHostToDevice));
    GF_TRY(dalloc_n(eng, &eng->es_nyq_idx, (size_t)n21));
    GF_TRY(dalloc_n(eng, &eng->es_nyq_op, std::max<size_t>(NOP.size(), 36)));
    GF_CU(cudaMemcpy(eng->es_nyq_idx, NIDX.data(), sizeof(int) * NIDX.size(), cudaMemcpyHostToDevice));
    if (!NOP.empty()) GF_CU(cudaMemcpy(eng->es_nyq_op, NOP.data(), sizeof(double) * NOP.size(), cudaMemcpyHostToDevice));
    int dimsi[3] = {P.nx, P.ny, P.nz};
    GF_FFT(cufftPlanMany(&eng->es_r2c, 3, dimsi, nullptr, 1, (int)n, nullptr, 1, (int)n21, CUFFT_D2Z, 6));
    GF_FFT(cufftPlanMany(&eng->es_c2r, 3, dimsi, nullptr, 1, (int)n21, nullptr, 1, (int)n, CUFFT_Z2D, 6));
    eng->es_plans = true;
    GF_FFT(cufftSetStream(eng->es_r2c, eng->stream));
    GF_FFT(cufftSetStream(eng->es_c2r, eng->stream));
    for (int a = 0; a < 6; a++) {
        if (!eng->es_eps[a]) GF_TRY(dalloc_r(eng, &eng->es_eps[a], (size_t)n));
        if (!eng->es_eig[a]) GF_TRY(dalloc_r(eng, &eng->es_eig[a], (size_t)n));
    }
    return GF_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// The reference's text outputs (inoutput.cpp:330-887, scheduled by
// main.cpp:170-198 and 486-705): the same file names, row order and printf
// formats (the file format is the interface a drop-in keeps), from fields
// downloaded in FP64.
// ---------------------------------------------------------------------------
namespace {

// a field in FP64 host memory; zeros when the run lacks it
int out_field(gf_engine* eng, int field, std::vector<double>& v) {
    size_t count = 0;
    GF_TRY(gf_field_dims(eng, field, nullptr, &count));
    v.assign(count, 0.);
    std::vector<double*> ptrs, cmps; std::vector<long> lens; bool writable, native;
    const std::string keep = eng->err;
    const int rc = field_ptrs(eng, field, ptrs, lens, writable, cmps, native);
    if (rc == GF_EINVAL || (rc == GF_OK && ptrs.empty())) {
        eng->err = keep;                 // absent in this run: the zeros stand
        return GF_OK;
    }
    GF_TRY(rc);
    return gf_download(eng, field, v.data(), count);
}

// "%ld  %ld  %ld  %.7e..." over a (nx_, ny_, nz_) grid, 1-based indices,
// component c of row (i, j, k) at cols[c][(i*ny_ + j)*nz_ + k]
int out_grid(gf_engine* eng, const std::string& path, long nx_, long ny_, long nz_, const std::vector<const double*>& cols) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) { eng->err = "cannot write " + path; return GF_EIO; }
    for (long i = 0; i < nx_; i++)
        for (long j = 0; j < ny_; j++)
            for (long k = 0; k < nz_; k++) {
                const long c = (i * ny_ + j) * nz_ + k;
                std::fprintf(f, "%ld  %ld  %ld", i + 1, j + 1, k + 1);
                for (const double* col : cols) std::fprintf(f, "  %.7e", col[c]);
                std::fprintf(f, "\n");
            }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    if (!ok) { eng->err = "write error in " + path; return GF_EIO; }
    return GF_OK;
}

// a cell field of ncomp components as "<name>.<nstep>.dat"
int out_cells(gf_engine* eng, const std::string& dir, const char* name, uint64_t nstep, int field) {
    std::vector<double> v;
    GF_TRY(out_field(eng, field, v));
    const long n = eng->P.n;
    std::vector<const double*> cols;
    for (size_t a = 0; a * (size_t)n < v.size(); a++) cols.push_back(v.data() + a * (size_t)n);
    return out_grid(eng, dir + "/" + name + "." + std::to_string(nstep) + ".dat", eng->P.nx, eng->P.ny, eng->P.nz, cols);
}

// a line appended to dir/name
int out_append(gf_engine* eng, const std::string& dir, const char* name, const std::string& line) {
    const std::string path = dir + "/" + name;
    FILE* f = std::fopen(path.c_str(), "a");
    if (!f) { eng->err = "cannot write " + path; return GF_EIO; }
    std::fputs(line.c_str(), f);
    std::fclose(f);
    return GF_OK;
}

// static strain in the global frame (exxt0_glb..), 6 x n; zeros without one
int out_static_strain_glb(gf_engine* eng, std::vector<double>& g) {
    std::vector<double> c;
    GF_TRY(out_field(eng, GF_FIELD_STRAIN_STATIC, c));
    const long n = eng->P.n;
    g.assign(6 * (size_t)n, 0.);
    const double(*T)[3] = eng->P.Tc2g;
    for (long q = 0; q < n; q++) {
        const double e[3][3] = {{c[0 * n + q], c[5 * n + q], c[4 * n + q]},
                                {c[5 * n + q], c[1 * n + q], c[3 * n + q]},
                                {c[4 * n + q], c[3 * n + q], c[2 * n + q]}};
        double r[3][3];
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                double s = 0.;
                for (int k = 0; k < 3; k++)
                    for (int l = 0; l < 3; l++) s += T[a][k] * T[b][l] * e[k][l];
                r[a][b] = s;
            }
        if (!eng->P.rot) std::memcpy(r, e, sizeof(r));
        g[0 * n + q] = r[0][0]; g[1 * n + q] = r[1][1]; g[2 * n + q] = r[2][2];
        g[3 * n + q] = r[1][2]; g[4 * n + q] = r[0][2]; g[5 * n + q] = r[0][1];
    }
    return GF_OK;
}

std::string out_line(const char* fmt, uint64_t nstep, const double* v, int nv) {
    char buf[256];
    if (nv == 3) std::snprintf(buf, sizeof(buf), fmt, (long long)nstep, v[0], v[1], v[2]);
    else std::snprintf(buf, sizeof(buf), fmt, (long long)nstep, v[0], v[1], v[2], v[3], v[4], v[5]);
    return buf;
}

int out_averages(gf_engine* eng, const std::string& dir, uint64_t nstep) {
    const Deck& d = eng->deck;
    double a[3], b[3];
    if (d.any_fm) {
        GF_TRY(gf_average(eng, GF_OBS_M, a));
        GF_TRY(out_append(eng, dir, "average_m.dat", out_line("%lld %.7e  %.7e  %.7e\n", nstep, a, 3)));
    }
    if (d.any_afm) {
        GF_TRY(gf_average(eng, GF_OBS_M_AFM1, a));
        GF_TRY(gf_average(eng, GF_OBS_M_AFM2, b));
        const double v[6] = {a[0], a[1], a[2], b[0], b[1], b[2]};
        GF_TRY(out_append(eng, dir, "average_AFMm.dat", out_line("%lld %.7e  %.7e  %.7e  %.7e  %.7e  %.7e\n", nstep, v, 6)));
    }
    if (d.any_fe) {
        GF_TRY(gf_average(eng, GF_OBS_P, a));
        GF_TRY(out_append(eng, dir, "average_p.dat", out_line("%lld %.7e  %.7e  %.7e\n", nstep, a, 3)));
    }
    return GF_OK;
}

bool out_due(const Deck::Out& o, uint64_t nstep) { return o.on && o.step > 0 && nstep % o.step == 0; }

}  // namespace

extern "C" {

int gf_create_from_deck(const char* deck_dir, int device, gf_engine** out) {
    return gf_create_from_deck_ex(deck_dir, device, GF_PRECISION_FP64, out);
}

int gf_create_from_deck_ex(const char* deck_dir, int device, int precision, gf_engine** out) {
    if (!deck_dir || !out) { g_create_err = "null argument"; return GF_EINVAL; }
    *out = nullptr;
    gf_engine* eng = new gf_engine();
    int rc = create(eng, deck_dir, device, precision);
    if (rc != GF_OK) {
        g_create_err = eng->err;
        gf_destroy(eng);
        return rc;
    }
    *out = eng;
    return GF_OK;
}

int gf_advance(gf_engine* e, uint64_t nsteps) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    GF_CU(cudaSetDevice(eng->device));
    return advance(e, nsteps, true);
}

int gf_create(const gf_run_params* run, const gf_material_params* mats, int n_materials, const uint32_t* material_cell,
              int device, int precision, gf_engine** out) {
    if (!run || !mats || !material_cell || !out) { g_create_err = "null argument"; return GF_EINVAL; }
    *out = nullptr;
    gf_engine* eng = new gf_engine();
    std::string e = deck_from_params(*run, mats, n_materials, material_cell, eng->deck);
    int rc = GF_OK;
    if (!e.empty()) { eng->err = e; rc = GF_EINVAL; }
    if (rc == GF_OK) rc = create_from(eng, "", device, precision);
    if (rc != GF_OK) {
        g_create_err = eng->err;
        gf_destroy(eng);
        return rc;
    }
    *out = eng;
    return GF_OK;
}

int gf_set_table(gf_engine* e, int table, const double* times, const double* xyz3, int64_t n) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (table != GF_TABLE_HEXT && table != GF_TABLE_EEXT) { eng->err = "unknown table"; return GF_EINVAL; }
    if (n < 0 || (n > 0 && (!times || !xyz3))) { eng->err = "bad table"; return GF_EINVAL; }
    Deck& d = eng->deck;
    const bool h = table == GF_TABLE_HEXT;
    if (!(h ? d.prescribe_H : d.prescribe_E)) {
        eng->err = h ? "the run has no prescribed H table (if_prescribe_Hext)" : "the run has no prescribed E table (if_prescribe_Eext)";
        return GF_EINVAL;
    }
    std::vector<double>& t = h ? d.tH : d.tE;
    std::vector<double>& x = h ? d.Hx : d.Ex;
    std::vector<double>& y = h ? d.Hy : d.Ey;
    std::vector<double>& z = h ? d.Hz : d.Ez;
    t.assign(times, times + n);
    x.resize(n); y.resize(n); z.resize(n);
    for (int64_t i = 0; i < n; i++) { x[i] = xyz3[3 * i]; y[i] = xyz3[3 * i + 1]; z[i] = xyz3[3 * i + 2]; }
    (h ? d.n_prescribe_H : d.n_prescribe_E) = (long)n;
    return GF_OK;
}

int gf_stage_begin(gf_engine* e, int stage) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (stage < 1 || stage > 4) { eng->err = "stage must be 1..4"; return GF_EINVAL; }
    if (eng->stage_open == 0) {
        if (stage != 1) { eng->err = "a step starts with stage 1"; return GF_EINVAL; }
        // time_marching_device_serial for the step: its drive row
        GF_CU(cudaSetDevice(eng->device));
        GF_CU(cudaStreamSynchronize(eng->stream));       // the pinned row buffer is free
        step_drive(eng, eng->drive_host[0]);
        const uint64_t slot = eng->steps_done & (uint64_t)(kDriveCap - 1);
        GF_CU(cudaMemcpyAsync(eng->drive + slot, eng->drive_host, sizeof(StepDrive), cudaMemcpyHostToDevice, eng->stream));
        eng->stage_open = 1;
        eng->stage_done = 0;
        return GF_OK;
    }
    // begin of the stage in progress (another system) or of the next one
    if (stage == eng->stage_done || stage == eng->stage_done + 1) return GF_OK;
    eng->err = "stage " + std::to_string(stage) + " begun after stage " + std::to_string(eng->stage_done);
    return GF_EINVAL;
}

int gf_stage_commit(gf_engine* e, int stage) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (stage < 1 || stage > 4) { eng->err = "stage must be 1..4"; return GF_EINVAL; }
    if (eng->stage_open == 0) {
        // a repeated commit of the stage that completed the last step
        if (stage == 4 && eng->stage_done == 4) return GF_OK;
        eng->err = "gf_stage_commit without gf_stage_begin";
        return GF_EINVAL;
    }
    if (stage == eng->stage_done) return GF_OK;               // served by the first commit
    if (stage != eng->stage_done + 1) {
        eng->err = "stage " + std::to_string(stage) + " committed after stage " + std::to_string(eng->stage_done);
        return GF_EINVAL;
    }
    GF_CU(cudaSetDevice(eng->device));
    const int parity = (int)(eng->steps_done & 1ull);
    if (eng->mixed) GF_TRY(gf_mixed_enqueue_stage(eng, parity, stage - 1));
    else GF_TRY(enqueue_stage_t<double>(eng, parity, stage - 1));
    eng->stage_done = stage;
    if (stage == 4) {
        GF_TRY(step_end(eng, parity, false));
        GF_CU(launch(k_step_inc, dim3(1), dim3(1), 0, eng->stream, eng->step_ctr));
        eng->steps_done += 1;
        eng->stage_open = 0;       // stage_done stays 4 until the next step begins
    }
    return GF_OK;
}

int gf_static_solve(gf_engine* e, int which) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    GF_CU(cudaSetDevice(eng->device));
    if (which != GF_STATIC_MAGNETIC && which != GF_STATIC_ELECTRIC) { eng->err = "unknown static solve"; return GF_EINVAL; }
    // between stages (main.cpp:299-306 and its repetitions) the committed
    // stage has already formed the static field of its new state
    if (eng->stage_done >= 1) return GF_OK;
    if (which == GF_STATIC_MAGNETIC) {
        if (eng->demag_mode < 0) { eng->err = "the run has no magnetostatics"; return GF_EINVAL; }
        if (eng->mixed) GF_TRY(demag_solve_f32(eng, f3f(cur(eng, eng->m)), f3f(cur(eng, eng->a1)), f3f(cur(eng, eng->a2)), false));
        else GF_TRY(demag_solve(eng, f3(cur(eng, eng->m)), f3(cur(eng, eng->a1)), f3(cur(eng, eng->a2)), false));
    } else if (which == GF_STATIC_ELECTRIC) {
        // with the solve off E_stat stays as it is, as in a build of the
        // reference's public sources, where get_E_static has no definition
        if (!eng->elec_on) return GF_OK;
        if (eng->elec_1d) GF_TRY(elec_1d_now(eng, (int)(eng->steps_done & 1ull)));
        else GF_TRY(elec_solve(eng, f3(cur(eng, eng->p)), false, eng->elec_iters, 0., nullptr));
    } else {
        eng->err = "unknown static solve";
        return GF_EINVAL;
    }
    GF_CU(cudaStreamSynchronize(eng->stream));
    return GF_OK;
}

int gf_advance_eager(gf_engine* e, uint64_t nsteps) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    GF_CU(cudaSetDevice(eng->device));
    return advance(e, nsteps, false);
}

int gf_average(gf_engine* e, int obs, double out3[3]) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!out3) { eng->err = "null output"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    double* const* src = nullptr;
    const Field3* f = nullptr;
    double denom = 1.;
    switch (obs) {
        case GF_OBS_M: if (!eng->m.on) break; f = &eng->m; src = cur(eng, eng->m); denom = (double)eng->deck.NFM; break;
        case GF_OBS_M_AFM1: if (!eng->a1.on) break; f = &eng->a1; src = cur(eng, eng->a1); denom = (double)eng->deck.NAFM; break;
        case GF_OBS_M_AFM2: if (!eng->a2.on) break; f = &eng->a2; src = cur(eng, eng->a2); denom = (double)eng->deck.NAFM; break;
        case GF_OBS_P: if (!eng->p.on) break; f = &eng->p; src = cur(eng, eng->p); denom = (double)eng->deck.NFE; break;
        case GF_OBS_U: if (!eng->u.on) break; f = &eng->u; src = cur(eng, eng->u); denom = (double)eng->P.n; break;
        default: break;
    }
    if (!src) { eng->err = "observable " + std::to_string(obs) + " is not present in this run"; return GF_EINVAL; }
    double s[3];
    GF_TRY(device_sum3(eng, src, eng->P.n, s, f->C));
    for (int a = 0; a < 3; a++) out3[a] = s[a] / denom;
    return GF_OK;
}

int gf_probe_em(gf_engine* e, int64_t i, int64_t j, int64_t k, double e3[3], double h3[3]) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    const Params& P = eng->P;
    if (!eng->E.on) { eng->err = "no Maxwell fields in this run"; return GF_EINVAL; }
    if (i < 0 || j < 0 || k < 0 || i >= P.nx || j >= P.ny || k >= P.nz) { eng->err = "probe outside the grid"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    // only the probed cell is centred
    const long c = (i * P.ny + j) * P.nz + k;
    GF_TRY(em_cells(eng, c, 1));
    for (int a = 0; a < 3; a++) GF_CU(cudaMemcpyAsync(&e3[a], eng->scratch + a * P.n + c, sizeof(double), cudaMemcpyDeviceToHost, eng->stream));
    double* hb = eng->scratch + 3 * P.n;
    for (int a = 0; a < 3; a++) GF_CU(cudaMemcpyAsync(&h3[a], hb + a * P.n + c, sizeof(double), cudaMemcpyDeviceToHost, eng->stream));
    GF_CU(cudaStreamSynchronize(eng->stream));
    return GF_OK;
}

int gf_field_dims(gf_engine* e, int field, int64_t dims3[3], size_t* count) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    const Params& P = eng->P;
    int64_t dx = P.nx, dy = P.ny, dz = P.nz;
    size_t ncomp = 3;
    if (field >= GF_FIELD_EX && field <= GF_FIELD_EZ) { int c = field - GF_FIELD_EX; dx += (c != 0); dy += (c != 1); dz += (c != 2); ncomp = 1; }
    else if (field >= GF_FIELD_HX && field <= GF_FIELD_HZ) { int c = field - GF_FIELD_HX; dx += (c == 0); dy += (c == 1); dz += (c == 2); ncomp = 1; }
    else if (field == GF_FIELD_STRAIN || field == GF_FIELD_STRAIN_STATIC || field == GF_FIELD_EIGENSTRAIN_STATIC) ncomp = 6;
    else if (field < 0 || field >= GF_FIELD_COUNT) { eng->err = "unknown field"; return GF_EINVAL; }
    if (dims3) { dims3[0] = dx; dims3[1] = dy; dims3[2] = dz; }
    if (count) *count = ncomp * (size_t)(dx * dy * dz);
    return GF_OK;
}

static int copy_field(gf_engine* eng, int field, double* buf, size_t count, bool to_host_or_dev_out, cudaMemcpyKind kind, bool sync) {
    std::vector<double*> ptrs, cmps; std::vector<long> lens; bool writable, native;
    GF_TRY(field_ptrs(eng, field, ptrs, lens, writable, cmps, native));
    size_t total = 0;
    for (long l : lens) total += (size_t)l;
    if (count != total) { eng->err = "field " + std::to_string(field) + " holds " + std::to_string(total) + " doubles, caller gave " + std::to_string(count); return GF_EINVAL; }
    if (!to_host_or_dev_out && !writable) { eng->err = "field is read-only"; return GF_EINVAL; }
    if (!to_host_or_dev_out && field == GF_FIELD_ESTAT) mark_estat(eng);
    const bool convert = eng->mixed && native;   // FP32 state <-> FP64 caller buffer through the scratch buffer
    size_t off = 0;
    for (size_t a = 0; a < ptrs.size(); a++) {
        const long len = lens[a];
        float* x = reinterpret_cast<float*>(ptrs[a]);
        float* cm = reinterpret_cast<float*>(cmps[a]);
        if (to_host_or_dev_out) {
            if (convert) {
                GF_CU(launch(k_widen, dim3(blocks_for(len, kThreads)), dim3(kThreads), 0, eng->stream, (const float*)x, (const float*)cm, len, eng->scratch));
                GF_CU(cudaMemcpyAsync(buf + off, eng->scratch, sizeof(double) * len, kind, eng->stream));
            } else {
                GF_CU(cudaMemcpyAsync(buf + off, ptrs[a], sizeof(double) * len, kind, eng->stream));
            }
        } else {
            if (convert) {
                GF_CU(cudaMemcpyAsync(eng->scratch, buf + off, sizeof(double) * len, kind, eng->stream));
                GF_CU(launch(k_split, dim3(blocks_for(len, kThreads)), dim3(kThreads), 0, eng->stream, (const double*)eng->scratch, len, x, cm));
            } else {
                GF_CU(cudaMemcpyAsync(ptrs[a], buf + off, sizeof(double) * len, kind, eng->stream));
            }
        }
        off += (size_t)len;
    }
    if (sync) GF_CU(cudaStreamSynchronize(eng->stream));
    return GF_OK;
}

int gf_download(gf_engine* e, int field, double* host, size_t count) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!host) { eng->err = "null buffer"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    return copy_field(e, field, host, count, true, cudaMemcpyDeviceToHost, true);
}

// A magnetisation given before the first step stands for the restart file the
// reference reads at set-up (m.in, m_AFM.in): the static field it computes
// from it before the time loop (main.cpp:135-146) is formed again from the
// uploaded state, unless the deck supplies Hstat.in.
static int after_upload(gf_engine* eng, int field) {
    GF_TRY(replicate_state(eng));
    const bool mag = field == GF_FIELD_M || field == GF_FIELD_M_AFM1 || field == GF_FIELD_M_AFM2;
    if (mag && eng->steps_done == 0 && !eng->deck.in_Hstat) {
        GF_TRY(static_field_now(eng));
        GF_CU(cudaStreamSynchronize(eng->stream));
    }
    return GF_OK;
}

int gf_upload(gf_engine* e, int field, const double* host, size_t count) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!host) { eng->err = "null buffer"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    GF_TRY(copy_field(e, field, const_cast<double*>(host), count, false, cudaMemcpyHostToDevice, true));
    return after_upload(e, field);
}

int gf_download_device(gf_engine* e, int field, double* dev, size_t count) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!dev) { eng->err = "null buffer"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    return copy_field(e, field, dev, count, true, cudaMemcpyDeviceToDevice, false);
}

int gf_upload_device(gf_engine* e, int field, const double* dev, size_t count) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!dev) { eng->err = "null buffer"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    GF_TRY(copy_field(e, field, const_cast<double*>(dev), count, false, cudaMemcpyDeviceToDevice, false));
    return after_upload(e, field);
}

// ---------------------------------------------------------------------------
// Checkpoint / restart (gf_save_state, gf_load_state)
// ---------------------------------------------------------------------------
struct CkBlob { std::string name; void* dev; size_t bytes; };

constexpr char kCkMagic[8] = {'G', 'F', 'B', '2', 'C', 'K', 'P', '1'};
struct CkHeader {
    char magic[8];
    int32_t nx, ny, nz, precision;
    uint64_t steps_done;
    double t_host;
    int64_t presc_H, presc_E;
    double Hext_cur[3], Eext_cur[3];
    uint32_t nblobs, reserved;
};

// every device array whose contents carry from one step to the next
std::vector<CkBlob> ck_blobs(gf_engine* eng) {
    std::vector<CkBlob> v;
    struct NF { const char* name; Field3* f; };
    NF fs[] = {{"m", &eng->m}, {"m_afm1", &eng->a1}, {"m_afm2", &eng->a2}, {"p", &eng->p}, {"q", &eng->q},
               {"u", &eng->u}, {"v", &eng->v}, {"E", &eng->E}, {"H", &eng->H},
               {"jp0", &eng->jp[0]}, {"jp1", &eng->jp[1]}, {"jp2", &eng->jp[2]}};
    for (const NF& nf : fs) {
        if (!nf.f->on) continue;
        double* const* c = cur(eng, *nf.f);
        for (int a = 0; a < 3; a++) {
            v.push_back({std::string(nf.name) + "." + std::to_string(a), c[a], eng->esz * (size_t)nf.f->len[a]});
            if (eng->mixed && nf.f->C[a])
                v.push_back({std::string(nf.name) + ".c" + std::to_string(a), nf.f->C[a], eng->esz * (size_t)nf.f->len[a]});
        }
    }
    const size_t n = (size_t)eng->P.n;
    for (int a = 0; a < 3; a++) {
        if (eng->Hstat[a]) v.push_back({"Hstat." + std::to_string(a), eng->Hstat[a], eng->esz * n});
        if (eng->Estat[a]) v.push_back({"Estat." + std::to_string(a), eng->Estat[a], eng->esz * n});
        if (eng->force_store[a]) v.push_back({"force_store." + std::to_string(a), eng->force_store[a], eng->esz * n});
    }
    const size_t plane = (size_t)eng->P.nx * eng->P.ny;
    if (eng->liao_hist) v.push_back({"liao_hist", eng->liao_hist, eng->esz * 4 * 12 * plane});
    if (eng->liao_last) v.push_back({"liao_last", eng->liao_last, eng->esz * 3 * plane});
    // static strain and eigenstrain, and the elastostatic solver's FP64
    // iterate (the start of the next per-step solve)
    for (int a = 0; a < 6; a++) {
        if (eng->es_eps[a]) v.push_back({"es_eps." + std::to_string(a), eng->es_eps[a], eng->esz * n});
        if (eng->es_eig[a]) v.push_back({"es_eig." + std::to_string(a), eng->es_eig[a], eng->esz * n});
    }
    if (eng->es_x) v.push_back({"es_x", eng->es_x, sizeof(double) * 6 * n});
    return v;
}

int gf_set_elastostatics(gf_engine* e, int enable, int* iterations_used) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    const Deck& d = eng->deck;
    if (iterations_used) *iterations_used = 0;
    if (!enable) {
        eng->es_on = false;
    } else {
        if (d.flexo && eng->P.flexo) {
            eng->err = "elastostatics with flexoelectricity (static-strain gradients) is not supported";
            return GF_EUNSUPPORTED;
        }
        GF_CU(cudaSetDevice(eng->device));
        GF_CU(cudaStreamSynchronize(eng->stream));
        GF_TRY(es_setup(eng));
        // the kernels read the static arrays through their stage inputs
        build_io(eng);
        if (eng->mixed) build_io_mixed(eng);
        const int limit = d.elasto_limit > 0 ? (int)d.elasto_limit : 500;
        const double tol = d.elasto_tol > 0. ? d.elasto_tol : 1e-10;
        eng->es_iters = limit;
        eng->es_per_step = !d.elastodynamics;
        int used = 0;
        GF_TRY(es_solve(eng, (int)(eng->steps_done & 1ull), false, limit, tol, &used));
        if (iterations_used) *iterations_used = used;
        GF_CU(cudaStreamSynchronize(eng->stream));
        eng->es_on = true;
    }
    invalidate_graphs(eng);
    return GF_OK;
}

int gf_set_electrostatics(gf_engine* e, int enable, int* iterations_used) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    const Deck& d = eng->deck;
    const Params& P = eng->P;
    if (iterations_used) *iterations_used = 0;
    if (!enable) {
        eng->elec_on = false;
        eng->elec_1d = false;
    } else {
        if (!d.any_fe) { eng->err = "electrostatics needs a ferroelectric material"; return GF_EINVAL; }
        GF_CU(cudaSetDevice(eng->device));
        GF_CU(cudaStreamSynchronize(eng->stream));
        if (d.elec_1D) {
            // the 1-D model (gf_elasto.cuh): P_z(t0) of the compensated form
            // is the polarisation now
            const int par = (int)(eng->steps_done & 1ull);
            if (d.elec_1D_comp) {
                if (!eng->elec_pz_t0) GF_TRY(dalloc_r(eng, &eng->elec_pz_t0, (size_t)P.n));
                GF_CU(cudaMemcpyAsync(eng->elec_pz_t0, cur(eng, eng->p)[2], eng->esz * (size_t)P.n, cudaMemcpyDeviceToDevice,
                                      eng->stream));
            }
            eng->elec_1d = true;
            eng->elec_on = true;
            eng->elec_per_stage = !d.em_dynamic;
            mark_estat(eng);
            if (!d.in_Estat) GF_TRY(elec_1d_now(eng, par));
            GF_CU(cudaStreamSynchronize(eng->stream));
            invalidate_graphs(eng);
            return GF_OK;
        }
        if (eng->mixed) { eng->err = "the spectral electrostatic solver runs in the FP64 form"; return GF_EUNSUPPORTED; }
        const long n21 = (long)P.nx * P.ny * (P.nz / 2 + 1);
        if (!eng->elec_q) {
            // wave vectors of global.cpp:276-316
            const double PI = kPi;
            const long dims[3] = {P.nx, P.ny, P.nz};
            const double h[3] = {P.dx, P.dy, P.dz};
            for (int a = 0; a < 3; a++) {
                const long len = (a < 2) ? dims[a] : dims[2] / 2 + 1;
                std::vector<double> kv((size_t)len);
                const double dk = 2. * PI / (static_cast<double>(dims[a]) * h[a]);
                for (long i = 0; i < len; i++) {
                    long t = i;
                    if (t > dims[a] / 2) t = t - dims[a];
                    kv[(size_t)i] = static_cast<double>(t) * dk;
                }
                GF_TRY(dalloc_n(eng, &eng->elec_k[a], (size_t)len));
                GF_CU(cudaStreamSynchronize(eng->stream));
                GF_CU(cudaMemcpy(eng->elec_k[a], kv.data(), sizeof(double) * len, cudaMemcpyHostToDevice));
            }
            GF_TRY(dalloc_n(eng, &eng->elec_q, (size_t)3 * P.n));
            GF_TRY(dalloc_n(eng, &eng->elec_qk, (size_t)3 * n21));
            GF_TRY(dalloc_n(eng, &eng->elec_blockmax, (size_t)2 * kElecBlocks));
            int dimsi[3] = {P.nx, P.ny, P.nz};
            GF_FFT(cufftPlanMany(&eng->elec_r2c, 3, dimsi, nullptr, 1, (int)P.n, nullptr, 1, (int)n21, CUFFT_D2Z, 3));
            GF_FFT(cufftPlanMany(&eng->elec_c2r, 3, dimsi, nullptr, 1, (int)n21, nullptr, 1, (int)P.n, CUFFT_Z2D, 3));
            eng->elec_plans = true;
            GF_FFT(cufftSetStream(eng->elec_r2c, eng->stream));
            GF_FFT(cufftSetStream(eng->elec_c2r, eng->stream));
        }
        // er_homo = max over materials of er, times scale_elec
        // (ferroelectric_initialize.cpp:310-318)
        double erh = d.mats[0].er;
        for (const Material& m : d.mats) erh = std::max(erh, m.er);
        eng->elec_erh = erh * (d.scale_elec > 0. ? d.scale_elec : 1.);
        const int limit = d.elec_limit > 0 ? (int)d.elec_limit : 200;
        const double tol = d.elec_tol > 0. ? d.elec_tol : 1e-12;
        eng->elec_iters = limit;
        eng->elec_on = true;
        mark_estat(eng);
        eng->elec_per_stage = !d.em_dynamic;
        // set-up solve from the current polarisation unless Estat.in was given
        // (main.cpp:122-131); it starts from the current E_stat
        if (!d.in_Estat) {
            int used = 0;
            GF_TRY(elec_solve(eng, f3(cur(eng, eng->p)), false, limit, tol, &used));
            if (iterations_used) *iterations_used = used;
        }
        GF_CU(cudaStreamSynchronize(eng->stream));
    }
    // the captured steps change
    for (int p = 0; p < 2; p++) {
        if (eng->gexec[p]) { cudaGraphExecDestroy(eng->gexec[p]); eng->gexec[p] = nullptr; }
        if (eng->graph[p]) { cudaGraphDestroy(eng->graph[p]); eng->graph[p] = nullptr; }
    }
    eng->graphs_ready = false;
    return GF_OK;
}

int gf_write_outputs(gf_engine* e, const char* dir, int initial) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!dir) { eng->err = "gf_write_outputs: null directory"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    const Deck& d = eng->deck;
    const Params& P = eng->P;
    const std::string D(dir);
    const uint64_t ns = eng->steps_done;
    const long n = P.n;
    if (initial) {
        // main.cpp:170-198
        if (d.out_ave.on) GF_TRY(out_averages(eng, D, ns));
        if (d.out_Estat.on) GF_TRY(out_cells(eng, D, "Estat", ns, GF_FIELD_ESTAT));
        if (d.out_Hstat.on) GF_TRY(out_cells(eng, D, "Hstat", ns, GF_FIELD_HSTAT));
        if (d.elastodynamics && d.out_strain.on) {
            std::vector<double> g;
            GF_TRY(out_static_strain_glb(eng, g));
            std::vector<const double*> cols;
            for (int a = 0; a < 6; a++) cols.push_back(g.data() + (size_t)a * n);
            GF_TRY(out_grid(eng, D + "/strain_stat." + std::to_string(ns) + ".dat", P.nx, P.ny, P.nz, cols));
        }
        if (d.out_eig0.on) GF_TRY(out_cells(eng, D, "eigenstraint0_crt", ns, GF_FIELD_EIGENSTRAIN_STATIC));
        return GF_OK;
    }
    // main.cpp:601-705, in its order
    if (out_due(d.out_ave, ns)) GF_TRY(out_averages(eng, D, ns));
    if (out_due(d.out_m, ns)) GF_TRY(out_cells(eng, D, "m", ns, GF_FIELD_M));
    if (out_due(d.out_magcell, ns)) {
        std::vector<double> m;
        GF_TRY(out_field(eng, GF_FIELD_M, m));
        const std::string path = D + "/m_magcell." + std::to_string(ns) + ".dat";
        FILE* f = std::fopen(path.c_str(), "w");
        if (!f) { eng->err = "cannot write " + path; return GF_EIO; }
        const long nyz = P.ny * P.nz;
        for (long c = 0; c < n; c++) {
            const uint8_t id = d.material_cell[(size_t)c];
            if (!(id && d.mats[id - 1].fm)) continue;
            const long i = c / nyz, j = (c - i * nyz) / P.nz, k = c - i * nyz - j * P.nz;
            std::fprintf(f, "%ld  %ld  %ld  %.7e  %.7e  %.7e\n", i + 1, j + 1, k + 1, m[c], m[n + c], m[2 * n + c]);
        }
        std::fclose(f);
    }
    if (out_due(d.out_AFMm, ns)) {
        std::vector<double> a1, a2;
        GF_TRY(out_field(eng, GF_FIELD_M_AFM1, a1));
        GF_TRY(out_field(eng, GF_FIELD_M_AFM2, a2));
        std::vector<const double*> cols;
        for (int a = 0; a < 3; a++) cols.push_back(a1.data() + (size_t)a * n);
        for (int a = 0; a < 3; a++) cols.push_back(a2.data() + (size_t)a * n);
        GF_TRY(out_grid(eng, D + "/m_AFM." + std::to_string(ns) + ".dat", P.nx, P.ny, P.nz, cols));
    }
    if (out_due(d.out_p, ns)) GF_TRY(out_cells(eng, D, "p", ns, GF_FIELD_P));
    if (out_due(d.out_q, ns)) GF_TRY(out_cells(eng, D, "q", ns, GF_FIELD_Q));
    if (out_due(d.out_em, ns)) {
        GF_TRY(out_cells(eng, D, "Eem", ns, GF_FIELD_E_CELL));
        GF_TRY(out_cells(eng, D, "Hem", ns, GF_FIELD_H_CELL));
    }
    if (out_due(d.out_em_onecell, ns)) {
        std::vector<double> E, H;
        GF_TRY(out_field(eng, GF_FIELD_E_CELL, E));
        GF_TRY(out_field(eng, GF_FIELD_H_CELL, H));
        const long c = (long)d.em_onecell_index - 1;
        if (c < 0 || c >= n) { eng->err = "em_onecell_index outside the grid"; return GF_EINVAL; }
        const double v[6] = {E[c], E[n + c], E[2 * n + c], H[c], H[n + c], H[2 * n + c]};
        GF_TRY(out_append(eng, D, "EM_onecell.dat", out_line("%lld %.7e  %.7e  %.7e %.7e  %.7e  %.7e\n", ns, v, 6)));
    }
    if (out_due(d.out_emYee, ns)) {
        const char* names[6] = {"Ex_Yee", "Ey_Yee", "Ez_Yee", "Hx_Yee", "Hy_Yee", "Hz_Yee"};
        for (int q = 0; q < 6; q++) {
            std::vector<double> v;
            GF_TRY(out_field(eng, GF_FIELD_EX + q, v));
            int64_t dm[3];
            GF_TRY(gf_field_dims(eng, GF_FIELD_EX + q, dm, nullptr));
            GF_TRY(out_grid(eng, D + "/" + names[q] + "." + std::to_string(ns) + ".dat", (long)dm[0], (long)dm[1], (long)dm[2],
                            {v.data()}));
        }
    }
    if (out_due(d.out_Estat, ns)) GF_TRY(out_cells(eng, D, "Estat", ns, GF_FIELD_ESTAT));
    if (out_due(d.out_Hstat, ns)) GF_TRY(out_cells(eng, D, "Hstat", ns, GF_FIELD_HSTAT));
    if (out_due(d.out_strain, ns)) {
        // static (global frame) plus dynamic cell strain, as output_strain
        // adds exxt0_glb and Dexx_glb
        std::vector<double> g, dyn;
        GF_TRY(out_static_strain_glb(eng, g));
        GF_TRY(out_field(eng, GF_FIELD_STRAIN, dyn));
        for (size_t q = 0; q < g.size(); q++) g[q] = g[q] + dyn[q];
        std::vector<const double*> cols;
        for (int a = 0; a < 6; a++) cols.push_back(g.data() + (size_t)a * n);
        GF_TRY(out_grid(eng, D + "/strain." + std::to_string(ns) + ".dat", P.nx, P.ny, P.nz, cols));
    }
    if (out_due(d.out_uv, ns)) {
        GF_TRY(out_cells(eng, D, "u", ns, GF_FIELD_U));
        GF_TRY(out_cells(eng, D, "v", ns, GF_FIELD_V));
    }
    if (out_due(d.out_force, ns)) GF_TRY(out_cells(eng, D, "elastoforce", ns, GF_FIELD_FORCE_STORE));
    if (out_due(d.out_eig0, ns)) GF_TRY(out_cells(eng, D, "eigenstraint0_crt", ns, GF_FIELD_EIGENSTRAIN_STATIC));
    if (out_due(d.out_Jp, ns)) {
        GF_TRY(out_cells(eng, D, "Jp1", ns, GF_FIELD_JP1));
        GF_TRY(out_cells(eng, D, "Jp2", ns, GF_FIELD_JP2));
        GF_TRY(out_cells(eng, D, "Jp3", ns, GF_FIELD_JP3));
    }
    return GF_OK;
}

int gf_run_deck(gf_engine* e, const char* dir) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    const Deck& d = eng->deck;
    GF_TRY(gf_write_outputs(e, dir, 1));
    const Deck::Out* outs[] = {&d.out_ave, &d.out_m, &d.out_magcell, &d.out_AFMm, &d.out_p, &d.out_q, &d.out_em,
                               &d.out_em_onecell, &d.out_emYee, &d.out_Estat, &d.out_Hstat, &d.out_strain, &d.out_uv,
                               &d.out_force, &d.out_eig0, &d.out_Jp};
    const uint64_t last = (uint64_t)d.steps;
    while (eng->steps_done < last) {
        uint64_t next = last;
        for (const Deck::Out* o : outs)
            if (o->on && o->step > 0) next = std::min<uint64_t>(next, (uint64_t)((eng->steps_done / o->step + 1) * o->step));
        GF_TRY(gf_advance(e, next - eng->steps_done));
        GF_TRY(gf_write_outputs(e, dir, 0));
    }
    return GF_OK;
}

int gf_save_state(gf_engine* e, const char* path) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!path) { eng->err = "null path"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    GF_CU(cudaStreamSynchronize(eng->stream));
    std::vector<CkBlob> blobs = ck_blobs(eng);
    CkHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kCkMagic, 8);
    h.nx = eng->P.nx; h.ny = eng->P.ny; h.nz = eng->P.nz;
    h.precision = eng->mixed ? GF_PRECISION_MIXED_FP32 : GF_PRECISION_FP64;
    h.steps_done = eng->steps_done; h.t_host = eng->t_host;
    h.presc_H = eng->presc_H; h.presc_E = eng->presc_E;
    for (int a = 0; a < 3; a++) { h.Hext_cur[a] = eng->Hext_cur[a]; h.Eext_cur[a] = eng->Eext_cur[a]; }
    h.nblobs = (uint32_t)blobs.size();
    FILE* f = std::fopen(path, "wb");
    if (!f) { eng->err = std::string("cannot write ") + path; return GF_EIO; }
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    std::vector<char> buf;
    for (const CkBlob& b : blobs) {
        if (!ok) break;
        char name[32];
        std::memset(name, 0, sizeof(name));
        std::strncpy(name, b.name.c_str(), sizeof(name) - 1);
        const uint64_t bytes = b.bytes;
        buf.resize(b.bytes);
        if (cudaMemcpy(buf.data(), b.dev, b.bytes, cudaMemcpyDeviceToHost) != cudaSuccess) { ok = false; break; }
        ok = std::fwrite(name, sizeof(name), 1, f) == 1 && std::fwrite(&bytes, sizeof(bytes), 1, f) == 1 &&
             std::fwrite(buf.data(), 1, b.bytes, f) == b.bytes;
    }
    if (std::fclose(f) != 0) ok = false;
    if (!ok) { eng->err = std::string("writing ") + path + " failed"; return GF_EIO; }
    return GF_OK;
}

int gf_load_state(gf_engine* e, const char* path) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!path) { eng->err = "null path"; return GF_EINVAL; }
    FILE* f = std::fopen(path, "rb");
    if (!f) { eng->err = std::string("cannot read ") + path; return GF_EIO; }
    CkHeader h;
    const unsigned long long steps_before = eng->steps_done;
    // the whole file is read and checked into host buffers before the first
    // device write, so a failed load leaves the engine as it was
    auto bad = [&](const std::string& why, int rc) { std::fclose(f); eng->err = why; eng->steps_done = steps_before; return rc; };
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kCkMagic, 8) != 0)
        return bad(std::string(path) + " is not an engine checkpoint", GF_EIO);
    if (h.nx != eng->P.nx || h.ny != eng->P.ny || h.nz != eng->P.nz)
        return bad("checkpoint grid differs from the engine's", GF_EINVAL);
    if (h.precision != (eng->mixed ? GF_PRECISION_MIXED_FP32 : GF_PRECISION_FP64))
        return bad("checkpoint precision differs from the engine's", GF_EINVAL);
    GF_CU(cudaSetDevice(eng->device));
    GF_CU(cudaStreamSynchronize(eng->stream));
    // the current-step buffers depend on the step parity: take the file's
    // (restored on failure by `bad`)
    eng->steps_done = h.steps_done;
    std::vector<CkBlob> blobs = ck_blobs(eng);
    if (h.nblobs != blobs.size()) return bad("checkpoint holds different fields than this engine", GF_EINVAL);
    std::vector<std::vector<char>> bufs(blobs.size());
    for (size_t q = 0; q < blobs.size(); q++) {
        const CkBlob& b = blobs[q];
        char name[32];
        uint64_t bytes = 0;
        if (std::fread(name, sizeof(name), 1, f) != 1 || std::fread(&bytes, sizeof(bytes), 1, f) != 1)
            return bad("truncated checkpoint", GF_EIO);
        name[31] = 0;
        if (b.name != name || bytes != b.bytes) return bad(std::string("checkpoint field ") + name + " does not match", GF_EINVAL);
        bufs[q].resize(bytes);
        if (std::fread(bufs[q].data(), 1, bytes, f) != bytes) return bad("truncated checkpoint", GF_EIO);
    }
    for (size_t q = 0; q < blobs.size(); q++)
        if (cudaMemcpy(blobs[q].dev, bufs[q].data(), blobs[q].bytes, cudaMemcpyHostToDevice) != cudaSuccess)
            return bad("checkpoint upload failed (device state now partly overwritten)", GF_ECUDA);
    std::fclose(f);
    eng->t_host = h.t_host; eng->presc_H = (long)h.presc_H; eng->presc_E = (long)h.presc_E;
    mark_estat(eng);     // the file's E_stat may be nonzero
    for (int a = 0; a < 3; a++) { eng->Hext_cur[a] = h.Hext_cur[a]; eng->Eext_cur[a] = h.Eext_cur[a]; }
    const unsigned long long ctr = h.steps_done;
    GF_CU(cudaMemcpy(eng->step_ctr, &ctr, sizeof(ctr), cudaMemcpyHostToDevice));
    return replicate_state(eng);
}

int gf_get_info(gf_engine* e, gf_info* info) {
    GF_TRY(check(e));
    if (!info) { e->err = "null info"; return GF_EINVAL; }
    const Deck& d = e->deck;
    std::memset(info, 0, sizeof(*info));
    info->nx = (int32_t)d.nx; info->ny = (int32_t)d.ny; info->nz = (int32_t)d.nz;
    info->dx = d.dx; info->dy = d.dy; info->dz = d.dz; info->dt = d.dt;
    info->time = e->t_host; info->step = e->steps_done; info->deck_steps = d.steps;
    info->n_materials = (int32_t)d.num_materials;
    info->fm = d.any_fm; info->afm = d.any_afm; info->fe = d.any_fe;
    info->elastic = d.elastodynamics; info->em = d.em_dynamic; info->demag_per_stage = e->demag_per_stage;
    info->n_fm = d.NFM; info->n_afm = d.NAFM; info->n_fe = d.NFE;
    info->device_bytes = e->bytes;
    info->launches_per_step = e->launches_per_step;
    info->precision = e->mixed ? GF_PRECISION_MIXED_FP32 : GF_PRECISION_FP64;
    return GF_OK;
}

int gf_profile_steps(gf_engine* e, uint64_t nsteps, gf_kernel_time* out, int max_records, int* n_records) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!out || !n_records || max_records <= 0) { eng->err = "null output"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    GF_CU(cudaStreamSynchronize(eng->stream));
    eng->profiling = true;
    eng->prof.clear();
    eng->ev_used = 0;
    int rc = advance(e, nsteps, false);
    eng->profiling = false;
    if (rc != GF_OK) return rc;
    GF_CU(cudaStreamSynchronize(eng->stream));
    int n = 0;
    for (auto& r : eng->prof) {
        float ms = 0.f;
        GF_CU(cudaEventElapsedTime(&ms, r.a, r.b));
        int slot = -1;
        for (int q = 0; q < n; q++) if (std::strncmp(out[q].name, r.name, sizeof(out[q].name)) == 0) { slot = q; break; }
        if (slot < 0) {
            if (n == max_records) continue;
            slot = n++;
            std::memset(&out[slot], 0, sizeof(out[slot]));
            std::strncpy(out[slot].name, r.name, sizeof(out[slot].name) - 1);
        }
        out[slot].launches += 1;
        out[slot].total_ms += (double)ms;
    }
    *n_records = n;
    eng->prof.clear();
    return GF_OK;
}

int gf_synchronize(gf_engine* e) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    GF_CU(cudaStreamSynchronize(eng->stream));
    return GF_OK;
}

void* gf_stream(gf_engine* e) { return e ? (void*)e->stream : nullptr; }

int gf_check_finite(gf_engine* e) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    GF_CU(cudaSetDevice(eng->device));
    struct Named { const char* name; Field3* f; };
    if (eng->tma_err) {
        unsigned h = 0;
        GF_CU(cudaMemcpyAsync(&h, eng->tma_err, sizeof(unsigned), cudaMemcpyDeviceToHost, eng->stream));
        GF_CU(cudaStreamSynchronize(eng->stream));
        if (h & 1u) { eng->err = "a TMA staging wait of the elastic tile timed out"; return GF_ECUDA; }
        if (h & 2u) { eng->err = "a grid barrier of the batch's persistent step timed out"; return GF_ECUDA; }
    }
    Named fs[] = {{"m", &eng->m}, {"m_afm1", &eng->a1}, {"m_afm2", &eng->a2}, {"p", &eng->p}, {"q", &eng->q}, {"u", &eng->u}, {"v", &eng->v}, {"E", &eng->E}, {"H", &eng->H}};
    for (auto& nf : fs) {
        if (!nf.f->on) continue;
        for (int a = 0; a < 3; a++) {
            GF_CU(cudaMemsetAsync(eng->flag, 0, sizeof(int), eng->stream));
            if (eng->mixed)
                GF_CU(launch(k_check_finite_f32, dim3(296), dim3(256), 0, eng->stream,
                             reinterpret_cast<const float*>(cur(eng, *nf.f)[a]), nf.f->len[a], eng->flag));
            else
                GF_CU(launch(k_check_finite, dim3(296), dim3(256), 0, eng->stream, (const double*)cur(eng, *nf.f)[a], nf.f->len[a], eng->flag));
            int h = 0;
            GF_CU(cudaMemcpyAsync(&h, eng->flag, sizeof(int), cudaMemcpyDeviceToHost, eng->stream));
            GF_CU(cudaStreamSynchronize(eng->stream));
            if (h) { eng->err = std::string("non-finite value in field ") + nf.name + " component " + std::to_string(a); return GF_ENAN; }
        }
    }
    return GF_OK;
}

const char* gf_last_error(const gf_engine* e) {
    if (!e) return g_create_err.c_str();
    return e->err.c_str();
}

void gf_destroy(gf_engine* e) {
    if (!e) return;
    if (e->stream) cudaStreamSynchronize(e->stream);
    for (int p = 0; p < 2; p++) {
        if (e->gexec[p]) cudaGraphExecDestroy(e->gexec[p]);
        if (e->graph[p]) cudaGraphDestroy(e->graph[p]);
    }
    if (e->plans) { cufftDestroy(e->plan_r2c); cufftDestroy(e->plan_c2r); }
    if (e->elec_plans) { cufftDestroy(e->elec_r2c); cufftDestroy(e->elec_c2r); }
    if (e->es_plans) { cufftDestroy(e->es_r2c); cufftDestroy(e->es_c2r); }
    for (cudaEvent_t ev : e->ev_pool) cudaEventDestroy(ev);
    for (void* p : e->allocs) cudaFree(p);
    if (e->drive_host) cudaFreeHost(e->drive_host);
    for (cudaStream_t b : e->side) if (b) cudaStreamDestroy(b);
    for (cudaEvent_t ev : e->bev) if (ev) cudaEventDestroy(ev);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

int gf_check_quotients(double d, uint64_t n, uint64_t seed, uint64_t* mismatches) {
    if (!mismatches || !(d != 0.) || !(d - d == 0.)) { g_create_err = "gf_check_quotients: need a finite nonzero d and an output"; return GF_EINVAL; }
    unsigned long long* bad = nullptr;
    cudaError_t ce = cudaMalloc(&bad, sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = cudaMemset(bad, 0, sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = launch(k_check_quotients, dim3(1184), dim3(256), 0, (cudaStream_t)0, d, 1. / d,
                                       (unsigned long long)n, (unsigned long long)seed, bad);
    unsigned long long h = 0;
    if (ce == cudaSuccess) ce = cudaMemcpy(&h, bad, sizeof(h), cudaMemcpyDeviceToHost);
    if (bad) cudaFree(bad);
    if (ce != cudaSuccess) { g_create_err = std::string("gf_check_quotients: ") + cudaGetErrorString(ce); return GF_ECUDA; }
    *mismatches = (uint64_t)h;
    return GF_OK;
}

const char* gf_version(void) { return "goferro_b200 0.2 (FP64 parity form, FP32 mixed form, sm_100a)"; }

}  // extern "C"


// ===========================================================================
// Batched runs (gf_batch_*): many engines advanced by one CUDA graph per step
//
// Each engine's step is captured as one branch of a single graph (fork and
// join events around the engines' own streams), so one graph launch advances
// every instance and instances of uneven grids run concurrently on the GPU.
// The autotuner picks, per engine, the x-chunk of the tiled elastic kernel
// (planes per block) from timed launches of that kernel on the engine's
// current state; the kernel writes only per-stage scratch, so tuning leaves
// every state untouched, and chunking does not change results.
// ===========================================================================
struct gf_batch {
    std::vector<gf_engine*> engs;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    std::string err;
    std::vector<int> tuned_chunk;
    // phase mode (mixed-form TDGL / elastodynamics / FDTD engines): one launch
    // per stage phase over the work items of every engine
    bool phases = false;
    bool split_tile = false;         // phase A as three concurrent launches (tile, Yee, TDGL items)
    std::vector<int> chunk;          // per engine: x-planes per elastic tile item
    BatchInst* dinst = nullptr;
    BatchItem* ditems[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};   // A (all), A tile, A Yee, A TDGL, B + C + D
    int nA = 0, nAt = 0, nAe = 0, nAf = 0, nB = 0, nC = 0, nD = 0;
    cudaStream_t side[2] = {nullptr, nullptr};   // split phase A: Yee and TDGL items beside the tile items
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    size_t smem = 0;
    // persistent mode: the whole step as one cooperative launch over the
    // phase mode's work lists, grid barriers between the phases
    bool persistent = false;
    unsigned* dbar = nullptr;        // barrier count and generation
    int pblocks = 0;                 // resident blocks of the launch
    std::string plan;
};

namespace {

#define GB_CU(call)                                                                      \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            b->err = std::string(#call) + ": " + cudaGetErrorString(e_);                 \
            return GF_ECUDA;                                                             \
        }                                                                                \
    } while (0)

int batch_fail(gf_batch* b, gf_engine* e, int rc) {
    b->err = std::string("engine: ") + (e ? e->err : std::string("?"));
    return rc;
}

// time the tile kernel at candidate chunks, keep the fastest
int autotune_tile(gf_batch* b, gf_engine* e) {
    const int nx = e->P.nx;
    const int base = e->el_chunk;
    std::vector<int> cand = {base};
    for (int L : {base / 2, base * 2, base * 4, (nx + 1) / 2, nx, 4, 8, 16})
        if (L >= 1 && L <= nx && std::find(cand.begin(), cand.end(), L) == cand.end()) cand.push_back(L);
    int best = base;
    float best_ms = -1.f;
    for (int L : cand) {
        e->el_chunk = L;
        float ms = 0.f;
        int rc = e->mixed ? gf_mixed_time_tile(e, 5, &ms) : time_tile_t<double>(e, 5, &ms);
        if (rc != GF_OK) { e->el_chunk = base; return batch_fail(b, e, rc); }
        if (best_ms < 0.f || ms < best_ms) { best_ms = ms; best = L; }
    }
    e->el_chunk = best;
    e->graphs_ready = false;          // the engine's own graphs hold the old grid
    for (int p = 0; p < 2; p++) {
        if (e->gexec[p]) { cudaGraphExecDestroy(e->gexec[p]); e->gexec[p] = nullptr; }
        if (e->graph[p]) { cudaGraphDestroy(e->graph[p]); e->graph[p] = nullptr; }
    }
    b->tuned_chunk.push_back(best);
    return GF_OK;
}

// Why engine e cannot run in the phase mode ("" if it can): the phase
// kernels cover the mixed form's TDGL, elastodynamics and Yee paths with Mur
// boundaries, without magnetism, flexoelectricity, static solves, plane
// sources, conductors or Drude poles.
std::string batch_phase_blocker(const gf_engine* e) {
    const Params& P = e->P;
    if (!e->mixed) return "FP64 engine";
    if (P.fm || P.afm) return "magnetic physics";
    if (P.flexo) return "flexoelectricity";
    if (P.planeEM || P.pec || P.drude) return "plane source, conductor or Drude poles";
    if (e->demag_mode >= 0 || e->elec_on || e->es_on) return "static solves";
    if (!(P.fe || P.em || P.elastic)) return "no stage kernels";
    return "";
}

// the work items of every engine at elastic x-chunk ch[i]: phase A's tile,
// Yee and TDGL items (A = all three, tiles first: the longest items); B the
// RK update, C the elastic boundary planes; an engine's Mur directions in
// order x, y, z in B, C, D, one phase each
void batch_items(const gf_batch* b, const std::vector<int>& ch, std::vector<BatchItem>& A, std::vector<BatchItem>& At,
                 std::vector<BatchItem>& Ae, std::vector<BatchItem>& Af, std::vector<BatchItem>& B, std::vector<BatchItem>& C,
                 std::vector<BatchItem>& D) {
    A.clear(); At.clear(); Ae.clear(); Af.clear(); B.clear(); C.clear(); D.clear();
    for (size_t i = 0; i < b->engs.size(); i++) {
        const Params& P = b->engs[i]->P;
        const int in = (int)i;
        const long nx = P.nx, ny = P.ny, nz = P.nz;
        if (P.elastic) {
            const int gx = (P.nz + etile::TK - 1) / etile::TK, gy = (P.ny + etile::TJ - 1) / etile::TJ;
            const int gz = (P.nx + ch[i] - 1) / ch[i];
            for (int z = 0; z < gz; z++)
                for (int y = 0; y < gy; y++)
                    for (int x = 0; x < gx; x++) At.push_back({in, BK_TILE, x, y, z});
            const int nrk = (int)blocks_for(P.n, 2 * kThreads);
            for (int x = 0; x < nrk; x++) B.push_back({in, BK_RK, x, 0, 0});
            const int nbc = P.el_bc_fused ? 0 : (int)blocks_for(nx * ny, kThreads);
            for (int x = 0; x < nbc; x++) C.push_back({in, BK_BC, x, 0, 0});
        }
        if (P.em) {
            const int gx = (int)blocks_for((ny + 1) * (nz + 1), kThreads);
            for (int y = 0; y <= P.nx; y++)
                for (int x = 0; x < gx; x++) Ae.push_back({in, BK_EM, x, y, 0});
            std::vector<BatchItem>* ph[3] = {&B, &C, &D};
            int q = 0;
            if (!P.per_x) { for (int x = 0; x < (int)blocks_for(ny * (nz + 1) + (ny + 1) * nz, kThreads); x++) ph[q]->push_back({in, BK_MUR_X, x, 0, 0}); q++; }
            if (!P.per_y) { for (int x = 0; x < (int)blocks_for(nx * (nz + 1) + (nx + 1) * nz, kThreads); x++) ph[q]->push_back({in, BK_MUR_Y, x, 0, 0}); q++; }
            if (!P.per_z) { for (int x = 0; x < (int)blocks_for(nx * (ny + 1) + (nx + 1) * ny, kThreads); x++) ph[q]->push_back({in, BK_MUR_Z, x, 0, 0}); q++; }
        }
        if (P.fe) {
            const int gx = (int)blocks_for(ny * nz, kThreads);
            for (int y = 0; y < P.nx; y++)
                for (int x = 0; x < gx; x++) Af.push_back({in, BK_FE, x, y, 0});
        }
    }
    A = At;
    A.insert(A.end(), Ae.begin(), Ae.end());
    A.insert(A.end(), Af.begin(), Af.end());
}

// device tables of the phase mode at chunks ch
int batch_upload(gf_batch* b, const std::vector<int>& ch) {
    std::vector<BatchInst> hi(b->engs.size());
    for (size_t i = 0; i < b->engs.size(); i++) {
        const gf_engine* e = b->engs[i];
        BatchInst& t = hi[i];
        std::memset(&t, 0, sizeof(t));
        t.P = e->P;
        for (int p = 0; p < 2; p++)
            for (int q = 0; q < 4; q++) t.io[p][q] = e->iof[p][q];
        t.cls = static_cast<const EmCls<float>*>(e->em_cls_tab);
        t.ncls = e->em_ncls;
        t.nmat = (int)e->deck.mats.size();
        t.el_chunk = ch[i];
        t.el_cubic = e->el_cubic ? 1 : 0;
        t.step = e->step_ctr;
    }
    std::vector<BatchItem> A, At, Ae, Af, B, C, D;
    batch_items(b, ch, A, At, Ae, Af, B, C, D);
    if (!b->dinst) GB_CU(cudaMalloc(&b->dinst, sizeof(BatchInst) * hi.size()));
    GB_CU(cudaMemcpy(b->dinst, hi.data(), sizeof(BatchInst) * hi.size(), cudaMemcpyHostToDevice));
    std::vector<BatchItem> BC = B;
    BC.insert(BC.end(), C.begin(), C.end());
    BC.insert(BC.end(), D.begin(), D.end());
    const std::vector<BatchItem>* L[5] = {&A, &At, &Ae, &Af, &BC};
    for (int q = 0; q < 5; q++) {
        if (b->ditems[q]) { cudaFree(b->ditems[q]); b->ditems[q] = nullptr; }
        if (!L[q]->empty()) {
            GB_CU(cudaMalloc(&b->ditems[q], sizeof(BatchItem) * L[q]->size()));
            GB_CU(cudaMemcpy(b->ditems[q], L[q]->data(), sizeof(BatchItem) * L[q]->size(), cudaMemcpyHostToDevice));
        }
    }
    b->nA = (int)A.size(); b->nAt = (int)At.size(); b->nAe = (int)Ae.size(); b->nAf = (int)Af.size();
    b->nB = (int)B.size(); b->nC = (int)C.size(); b->nD = (int)D.size();
    b->chunk = ch;
    return GF_OK;
}

#define GB_PH(call)                                                                        \
    do {                                                                                   \
        const int ce_ = (call);                                                            \
        if (ce_ != 0) {                                                                    \
            b->err = std::string("batch phase launch: ") + cudaGetErrorString((cudaError_t)ce_); \
            return GF_ECUDA;                                                               \
        }                                                                                  \
    } while (0)

// phase A of stage s: one launch, or the tile, Yee and TDGL items as three
// launches forked onto the batch's side streams and joined again
int batch_phase_a(gf_batch* b, int s, int parity, cudaStream_t st) {
    unsigned* err = b->engs[0]->tma_err;
    if (b->split_tile) {
        GB_CU(cudaEventRecord(b->ev[0], st));
        GB_CU(cudaStreamWaitEvent(b->side[0], b->ev[0], 0));
        GB_CU(cudaStreamWaitEvent(b->side[1], b->ev[0], 0));
        GB_PH(gf_mixed_batch_phase(b->dinst, b->ditems[1], b->nAt, s, 3, parity, b->smem, err, st));
        GB_PH(gf_mixed_batch_phase(b->dinst, b->ditems[2], b->nAe, s, 4, parity, b->smem, err, b->side[0]));
        GB_PH(gf_mixed_batch_phase(b->dinst, b->ditems[3], b->nAf, s, 5, parity, b->smem, err, b->side[1]));
        GB_CU(cudaEventRecord(b->ev[1], b->side[0]));
        GB_CU(cudaEventRecord(b->ev[2], b->side[1]));
        GB_CU(cudaStreamWaitEvent(st, b->ev[1], 0));
        GB_CU(cudaStreamWaitEvent(st, b->ev[2], 0));
        return GF_OK;
    }
    GB_PH(gf_mixed_batch_phase(b->dinst, b->ditems[0], b->nA, s, 0, parity, b->smem, err, st));
    return GF_OK;
}

// one step of every engine in the persistent mode: one cooperative launch
int batch_enqueue_persistent(gf_batch* b, int parity, cudaStream_t st) {
    GB_PH(gf_mixed_batch_persistent(b->dinst, (int)b->engs.size(), b->ditems[0], b->nA, b->ditems[4], b->nB, b->nC, b->nD, parity,
                                    b->smem, b->engs[0]->tma_err, b->dbar, b->pblocks, st));
    return GF_OK;
}

// one step of every engine in the phase mode: 4 stages x (A, B, C, D; the
// empty ones skipped), then
// the step counters
int batch_enqueue_phases(gf_batch* b, int parity, cudaStream_t st) {
    unsigned* err = b->engs[0]->tma_err;
    for (int s = 0; s < 4; s++) {
        GF_TRY(batch_phase_a(b, s, parity, st));
        if (b->nB > 0) GB_PH(gf_mixed_batch_phase(b->dinst, b->ditems[4], b->nB, s, 1, parity, 0, err, st));
        if (b->nC > 0) GB_PH(gf_mixed_batch_phase(b->dinst, b->ditems[4] + b->nB, b->nC, s, 1, parity, 0, err, st));
        if (b->nD > 0) GB_PH(gf_mixed_batch_phase(b->dinst, b->ditems[4] + b->nB + b->nC, b->nD, s, 1, parity, 0, err, st));
    }
    GB_CU(launch(k_batch_step_inc, dim3(blocks_for((long)b->engs.size(), kThreads)), dim3(kThreads), 0, st,
                 (const BatchInst*)b->dinst, (int)b->engs.size()));
    return GF_OK;
}

// mean device time of `reps` launches of one phase-A item list of stage 0
// (kind 3 tile, 4 Yee, 5 TDGL items)
int batch_time_kind(gf_batch* b, int ph, int reps, float* ms) {
    const int parity = (int)(b->engs[0]->steps_done & 1ull);
    const int q = ph - 2;
    const int n = ph == 3 ? b->nAt : (ph == 4 ? b->nAe : b->nAf);
    *ms = 0.f;
    if (n == 0) return GF_OK;
    cudaEvent_t e0, e1;
    GB_CU(cudaEventCreate(&e0));
    GB_CU(cudaEventCreate(&e1));
    int ce = gf_mixed_batch_phase(b->dinst, b->ditems[q], n, 0, ph, parity, b->smem, b->engs[0]->tma_err, b->stream);
    if (ce == 0) ce = (int)cudaEventRecord(e0, b->stream);
    for (int r = 0; r < reps && ce == 0; r++)
        ce = gf_mixed_batch_phase(b->dinst, b->ditems[q], n, 0, ph, parity, b->smem, b->engs[0]->tma_err, b->stream);
    if (ce == 0) ce = (int)cudaEventRecord(e1, b->stream);
    if (ce == 0) ce = (int)cudaEventSynchronize(e1);
    float t = 0.f;
    if (ce == 0) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (ce != 0) { b->err = std::string("batch kind timing: ") + cudaGetErrorString((cudaError_t)ce); return GF_ECUDA; }
    *ms = t / (float)(reps > 0 ? reps : 1);
    return GF_OK;
}

// mean device time of `reps` phase-A launches of stage 0 (they write stage-0
// outputs and per-stage scratch only: the state is not touched)
int batch_time_phase_a(gf_batch* b, int reps, float* ms) {
    const int parity = (int)(b->engs[0]->steps_done & 1ull);
    cudaEvent_t e0, e1;
    GB_CU(cudaEventCreate(&e0));
    GB_CU(cudaEventCreate(&e1));
    int rc = batch_phase_a(b, 0, parity, b->stream);
    if (rc == GF_OK && cudaEventRecord(e0, b->stream) != cudaSuccess) rc = GF_ECUDA;
    for (int r = 0; r < reps && rc == GF_OK; r++) rc = batch_phase_a(b, 0, parity, b->stream);
    if (rc == GF_OK && cudaEventRecord(e1, b->stream) != cudaSuccess) rc = GF_ECUDA;
    if (rc == GF_OK && cudaEventSynchronize(e1) != cudaSuccess) rc = GF_ECUDA;
    float t = 0.f;
    if (rc == GF_OK) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != GF_OK) { if (b->err.empty()) b->err = "batch phase timing"; return rc; }
    *ms = t / (float)(reps > 0 ? reps : 1);
    return GF_OK;
}

// The phase mode's autotuner: the elastic tile's x-chunk per work item (one
// chunk for every engine, capped at the engine's nx, or each engine's own
// one-engine choice) and whether phase A is one fused launch or the tile
// items and the others in two, from timed phase-A launches.
int batch_tune_phases(gf_batch* b, int autotune) {
    std::vector<int> own(b->engs.size());
    for (size_t i = 0; i < b->engs.size(); i++) own[i] = std::max(1, b->engs[i]->el_chunk);
    std::vector<std::vector<int>> cands = {own};
    if (autotune)
        for (int L : {2, 4, 8, 16, 32}) {
            std::vector<int> c(b->engs.size());
            for (size_t i = 0; i < b->engs.size(); i++) c[i] = std::min(L, b->engs[i]->P.nx);
            cands.push_back(c);
        }
    bool any_tile = false;
    for (gf_engine* e : b->engs) any_tile = any_tile || e->P.elastic;
    float best = -1.f;
    std::vector<int> best_c = own;
    bool best_split = false;
    std::string log;
    for (size_t ci = 0; ci < cands.size(); ci++) {
        if (!any_tile && ci > 0) break;
        GF_TRY(batch_upload(b, cands[ci]));
        for (int split = 0; split < ((autotune && any_tile) ? 2 : 1); split++) {
            b->split_tile = split != 0;
            float ms = 0.f;
            GF_TRY(batch_time_phase_a(b, autotune ? 3 : 0, &ms));
            if (!autotune) { best_c = cands[ci]; best_split = false; break; }
            char buf[96];
            std::snprintf(buf, sizeof(buf), "%s%s %s %.4f ms", log.empty() ? "" : "; ",
                          ci == 0 ? "own" : ("L=" + std::to_string(cands[ci][0])).c_str(), split ? "split" : "fused", ms);
            log += buf;
            if (best < 0.f || ms < best) { best = ms; best_c = cands[ci]; best_split = split != 0; }
        }
    }
    GF_TRY(batch_upload(b, best_c));
    b->split_tile = best_split;
    std::string kinds;
    if (autotune) {
        float tk[3] = {0.f, 0.f, 0.f};
        for (int q = 0; q < 3; q++) GF_TRY(batch_time_kind(b, 3 + q, 3, &tk[q]));
        char buf[128];
        std::snprintf(buf, sizeof(buf), "; alone at the chosen chunk: tile %.4f, Yee %.4f, TDGL %.4f ms", tk[0], tk[1], tk[2]);
        kinds = buf;
    }
    b->plan = "phases: " + std::to_string(b->engs.size()) + " engines, " + std::to_string(b->nA) + " phase-A, " +
              std::to_string(b->nB) + " phase-B, " + std::to_string(b->nC) + " phase-C, " + std::to_string(b->nD) +
              " phase-D items per stage; phase A " +
              (best_split ? "split (tile, Yee and TDGL items in three concurrent launches)" : "fused (tile, Yee and TDGL items in one launch)") +
              (autotune ? "; timed phase A (stage 1): " + log + kinds : std::string("; untuned (each engine's own chunk)"));
    return GF_OK;
}

// the step graphs (one per step parity) of the phase mode (phases) or the
// branch mode into g / gx
int batch_capture(gf_batch* b, bool phases, cudaGraph_t* gout, cudaGraphExec_t* gxout, bool persistent = false) {
    if (phases) {
        for (int par = 0; par < 2; par++) {
            GB_CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            const int rc = persistent ? batch_enqueue_persistent(b, par, b->stream) : batch_enqueue_phases(b, par, b->stream);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
            if (rc != GF_OK || ce != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                if (rc == GF_OK) b->err = std::string("batch capture: ") + cudaGetErrorString(ce);
                return rc != GF_OK ? rc : GF_ECUDA;
            }
            gout[par] = g;
            GB_CU(cudaGraphInstantiate(&gxout[par], g, 0));
        }
        return GF_OK;
    }
    for (int par = 0; par < 2; par++) {
        GB_CU(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int rc = GF_OK;
        cudaError_t ce = cudaEventRecord(b->fork, b->stream);
        for (size_t i = 0; i < b->engs.size() && rc == GF_OK && ce == cudaSuccess; i++) {
            gf_engine* e = b->engs[i];
            ce = cudaStreamWaitEvent(e->stream, b->fork, 0);
            if (ce == cudaSuccess) {
                rc = enqueue_step(e, par);
                if (rc != GF_OK) b->err = std::string("engine: ") + e->err;
            }
            if (rc == GF_OK && ce == cudaSuccess) ce = cudaEventRecord(b->join[i], e->stream);
            if (rc == GF_OK && ce == cudaSuccess) ce = cudaStreamWaitEvent(b->stream, b->join[i], 0);
        }
        cudaGraph_t g = nullptr;
        cudaError_t ce2 = cudaStreamEndCapture(b->stream, &g);
        if (rc != GF_OK || ce != cudaSuccess || ce2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            if (rc == GF_OK) b->err = std::string("batch capture: ") + cudaGetErrorString(ce != cudaSuccess ? ce : ce2);
            return rc != GF_OK ? rc : GF_ECUDA;
        }
        gout[par] = g;
        GB_CU(cudaGraphInstantiate(&gxout[par], g, 0));
    }
    return GF_OK;
}

// nsteps steps of every engine with the step graphs gx: the engines' drive
// rows uploaded per chunk, then one graph launch per step (events e0 / e1,
// when given, around the launches of the first chunk)
int batch_run(gf_batch* b, cudaGraphExec_t* gx, uint64_t nsteps, cudaEvent_t e0, cudaEvent_t e1) {
    uint64_t done = 0;
    while (done < nsteps) {
        const uint64_t chunk = std::min<uint64_t>(nsteps - done, (uint64_t)kDriveCap / 2);
        GB_CU(cudaStreamSynchronize(b->stream));
        for (gf_engine* e : b->engs) {
            for (uint64_t s = 0; s < chunk; s++) step_drive(e, e->drive_host[s]);
            const uint64_t first = e->steps_done + done;
            uint64_t s = 0;
            while (s < chunk) {
                const uint64_t slot = (first + s) & (uint64_t)(kDriveCap - 1);
                const uint64_t run = std::min<uint64_t>(chunk - s, (uint64_t)kDriveCap - slot);
                GB_CU(cudaMemcpyAsync(e->drive + slot, e->drive_host + s, sizeof(StepDrive) * run, cudaMemcpyHostToDevice, b->stream));
                s += run;
            }
        }
        const uint64_t first = b->engs[0]->steps_done + done;
        if (e0 && done == 0) GB_CU(cudaEventRecord(e0, b->stream));
        for (uint64_t k = 0; k < chunk; k++) GB_CU(cudaGraphLaunch(gx[(first + k) & 1ull], b->stream));
        if (e1 && done == 0) GB_CU(cudaEventRecord(e1, b->stream));
        done += chunk;
    }
    for (gf_engine* e : b->engs) e->steps_done += nsteps;
    return GF_OK;
}

// Every engine's step-to-step state (the checkpoint's device arrays, the
// device step counter, the host clock), kept on the device so that trial
// steps can be undone.
struct BatchSnap {
    struct Host { uint64_t steps_done; double t_host; long presc_H, presc_E; double Hext_cur[3], Eext_cur[3]; };
    std::vector<Host> host;
    std::vector<std::vector<CkBlob>> blobs;
    char* dev = nullptr;
    size_t bytes = 0;
};

int batch_snap_take(gf_batch* b, BatchSnap& sn) {
    sn.host.clear(); sn.blobs.clear(); sn.bytes = 0;
    for (gf_engine* e : b->engs) {
        sn.blobs.push_back(ck_blobs(e));
        sn.blobs.back().push_back({"step_ctr", e->step_ctr, sizeof(unsigned long long)});
        for (const CkBlob& c : sn.blobs.back()) sn.bytes += (c.bytes + 255) & ~(size_t)255;
        BatchSnap::Host h;
        h.steps_done = e->steps_done; h.t_host = e->t_host; h.presc_H = e->presc_H; h.presc_E = e->presc_E;
        std::memcpy(h.Hext_cur, e->Hext_cur, sizeof(h.Hext_cur)); std::memcpy(h.Eext_cur, e->Eext_cur, sizeof(h.Eext_cur));
        sn.host.push_back(h);
    }
    GB_CU(cudaMalloc(&sn.dev, sn.bytes));
    size_t off = 0;
    for (const auto& bl : sn.blobs)
        for (const CkBlob& c : bl) {
            GB_CU(cudaMemcpyAsync(sn.dev + off, c.dev, c.bytes, cudaMemcpyDeviceToDevice, b->stream));
            off += (c.bytes + 255) & ~(size_t)255;
        }
    GB_CU(cudaStreamSynchronize(b->stream));
    return GF_OK;
}

int batch_snap_put(gf_batch* b, const BatchSnap& sn) {
    GB_CU(cudaStreamSynchronize(b->stream));
    size_t off = 0;
    for (size_t i = 0; i < b->engs.size(); i++) {
        for (const CkBlob& c : sn.blobs[i]) {
            GB_CU(cudaMemcpyAsync(c.dev, sn.dev + off, c.bytes, cudaMemcpyDeviceToDevice, b->stream));
            off += (c.bytes + 255) & ~(size_t)255;
        }
        gf_engine* e = b->engs[i];
        const BatchSnap::Host& h = sn.host[i];
        e->steps_done = h.steps_done; e->t_host = h.t_host; e->presc_H = h.presc_H; e->presc_E = h.presc_E;
        std::memcpy(e->Hext_cur, h.Hext_cur, sizeof(h.Hext_cur)); std::memcpy(e->Eext_cur, h.Eext_cur, sizeof(h.Eext_cur));
    }
    GB_CU(cudaStreamSynchronize(b->stream));
    return GF_OK;
}

// device time per step of `steps` steps with graphs gx after two warm-up
// steps, the state restored before each run and at the end
int batch_trial(gf_batch* b, const BatchSnap& sn, cudaGraphExec_t* gx, int steps, float* ms) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GB_CU(cudaEventCreate(&e0));
    GB_CU(cudaEventCreate(&e1));
    int rc = batch_snap_put(b, sn);
    if (rc == GF_OK) rc = batch_run(b, gx, 2, nullptr, nullptr);
    if (rc == GF_OK) rc = batch_snap_put(b, sn);
    if (rc == GF_OK) rc = batch_run(b, gx, (uint64_t)steps, e0, e1);
    float t = 0.f;
    if (rc == GF_OK && cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
    if (rc == GF_OK) rc = batch_snap_put(b, sn);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms = t / (float)steps;
    return rc;
}

}  // namespace

extern "C" {

int gf_batch_create(gf_engine* const* engines, int count, int autotune, gf_batch** out) {
    return gf_batch_create_ex(engines, count, autotune, GF_BATCH_AUTO, out);
}

int gf_batch_create_ex(gf_engine* const* engines, int count, int autotune, int mode, gf_batch** out) {
    if (!engines || count < 1 || !out) { g_create_err = "gf_batch_create: need engines, count >= 1 and an output"; return GF_EINVAL; }
    if (mode != GF_BATCH_AUTO && mode != GF_BATCH_BRANCHES && mode != GF_BATCH_PHASES && mode != GF_BATCH_PERSISTENT)
        { g_create_err = "gf_batch_create_ex: unknown mode"; return GF_EINVAL; }
    *out = nullptr;
    gf_batch* b = new gf_batch();
    b->device = engines[0]->device;
    for (int i = 0; i < count; i++) {
        gf_engine* e = engines[i];
        if (!e) { g_create_err = "gf_batch_create: null engine"; delete b; return GF_EINVAL; }
        if (e->device != b->device) { g_create_err = "gf_batch_create: engines on different devices"; delete b; return GF_EINVAL; }
        if ((e->steps_done & 1ull) != (engines[0]->steps_done & 1ull)) {
            g_create_err = "gf_batch_create: engines must be at steps of the same parity"; delete b; return GF_EINVAL;
        }
        for (int j = 0; j < i; j++)
            if (engines[j] == e) { g_create_err = "gf_batch_create: an engine appears twice"; delete b; return GF_EINVAL; }
        b->engs.push_back(e);
    }
    auto fail = [&](int rc) { g_create_err = b->err; gf_batch_destroy(b); return rc; };
    if (cudaSetDevice(b->device) != cudaSuccess) { b->err = "cudaSetDevice"; return fail(GF_ECUDA); }
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) { b->err = "stream"; return fail(GF_ECUDA); }
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) { b->err = "event"; return fail(GF_ECUDA); }
    b->join.assign(b->engs.size(), nullptr);
    for (auto& ev : b->join)
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) { b->err = "event"; return fail(GF_ECUDA); }
    for (gf_engine* e : b->engs)
        if (cudaStreamSynchronize(e->stream) != cudaSuccess) { b->err = "engine stream"; return fail(GF_ECUDA); }
    std::string blocker;
    for (gf_engine* e : b->engs)
        if (blocker.empty()) blocker = batch_phase_blocker(e);
    if ((mode == GF_BATCH_PHASES || mode == GF_BATCH_PERSISTENT) && !blocker.empty())
        { b->err = "gf_batch_create_ex: phase mode: " + blocker; return fail(GF_EUNSUPPORTED); }
    b->phases = mode != GF_BATCH_BRANCHES && blocker.empty();
    // with GF_BATCH_AUTO and autotune, both modes are built and timed below
    const bool choose = b->phases && mode == GF_BATCH_AUTO && autotune;
    if (b->phases) {
        for (int q = 0; q < 2; q++)
            if (cudaStreamCreateWithFlags(&b->side[q], cudaStreamNonBlocking) != cudaSuccess) { b->err = "stream"; return fail(GF_ECUDA); }
        for (int q = 0; q < 3; q++)
            if (cudaEventCreateWithFlags(&b->ev[q], cudaEventDisableTiming) != cudaSuccess) { b->err = "event"; return fail(GF_ECUDA); }
        int nmat = 1;
        for (gf_engine* e : b->engs) nmat = std::max(nmat, (int)e->deck.mats.size());
        b->smem = batch_smem_bytes(nmat);
        if (gf_mixed_batch_attr(b->smem) != GF_OK) { b->err = "batch kernels: shared-memory attribute"; return fail(GF_ECUDA); }
        int rc = batch_tune_phases(b, autotune);
        if (rc != GF_OK) return fail(rc);
        if (cudaStreamSynchronize(b->stream) != cudaSuccess) { b->err = "batch tuning"; return fail(GF_ECUDA); }
        if (mode == GF_BATCH_PERSISTENT || choose) {
            // the persistent step's barrier and grid: every block resident
            if (cudaMalloc(&b->dbar, 2 * sizeof(unsigned)) != cudaSuccess || cudaMemset(b->dbar, 0, 2 * sizeof(unsigned)) != cudaSuccess)
                { b->err = "batch barrier"; return fail(GF_ECUDA); }
            if (gf_mixed_batch_persistent_blocks(b->smem, &b->pblocks) != GF_OK || b->pblocks < 1)
                { b->err = "batch persistent kernel: occupancy"; return fail(GF_ECUDA); }
        }
        b->persistent = mode == GF_BATCH_PERSISTENT;
        if (b->persistent) b->plan = "persistent: one cooperative launch per step over the " + b->plan.substr(8) +
                                     "; " + std::to_string(b->pblocks) + " resident blocks";
    }
    if (!b->phases || choose) {
        if (!b->phases)
            b->plan = "branches: one graph branch per engine" + (blocker.empty() ? std::string() : " (phase mode: " + blocker + ")");
        if (autotune)
            for (gf_engine* e : b->engs)
                if (e->P.elastic) {
                    int rc = autotune_tile(b, e);
                    if (rc != GF_OK) return fail(rc);
                }
    }
    int rc = batch_capture(b, b->phases, b->graph, b->gexec, b->persistent);
    if (rc != GF_OK) return fail(rc);
    if (choose) {
        // the fusion choice: one graph branch per engine, the phase
        // launches over all engines, or the persistent step, from timed
        // steps whose state is undone
        cudaGraph_t g2[2] = {nullptr, nullptr}, g3[2] = {nullptr, nullptr};
        cudaGraphExec_t gx2[2] = {nullptr, nullptr}, gx3[2] = {nullptr, nullptr};
        auto drop = [](cudaGraph_t* g, cudaGraphExec_t* x) {
            for (int p = 0; p < 2; p++) {
                if (x[p]) cudaGraphExecDestroy(x[p]);
                if (g[p]) cudaGraphDestroy(g[p]);
                x[p] = nullptr; g[p] = nullptr;
            }
        };
        rc = batch_capture(b, false, g2, gx2);
        // the persistent step: a capture the runtime refuses leaves it out
        std::string pnote;
        const std::string err0 = b->err;
        if (rc == GF_OK && batch_capture(b, true, g3, gx3, true) != GF_OK) {
            pnote = "; persistent step not captured (" + b->err + ")";
            b->err = err0;
            drop(g3, gx3);
            (void)cudaGetLastError();
        }
        BatchSnap sn;
        float t_ph = 0.f, t_br = 0.f, t_pe = -1.f;
        if (rc == GF_OK) rc = batch_snap_take(b, sn);
        if (rc == GF_OK) rc = batch_trial(b, sn, b->gexec, 4, &t_ph);
        if (rc == GF_OK) rc = batch_trial(b, sn, gx2, 4, &t_br);
        if (rc == GF_OK && gx3[0]) {
            rc = batch_trial(b, sn, gx3, 4, &t_pe);
            // a barrier that gave up leaves bit 2 of the flag: that step is
            // not a candidate (the trial's state is undone)
            unsigned h = 0;
            if (rc == GF_OK && cudaMemcpy(&h, b->engs[0]->tma_err, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess) rc = GF_ECUDA;
            if (rc == GF_OK && (h & 2u)) {
                pnote = "; persistent step: a grid barrier timed out, left out";
                t_pe = -1.f;
                const unsigned z = h & ~2u;
                if (cudaMemcpy(b->engs[0]->tma_err, &z, sizeof(unsigned), cudaMemcpyHostToDevice) != cudaSuccess) rc = GF_ECUDA;
            }
        }
        if (sn.dev) cudaFree(sn.dev);
        if (rc != GF_OK) { drop(g2, gx2); drop(g3, gx3); return fail(rc); }
        char buf[160];
        if (t_pe >= 0.f)
            std::snprintf(buf, sizeof(buf), "; timed steps: phases %.4f ms, branches %.4f ms, persistent %.4f ms (%d resident blocks)",
                          t_ph, t_br, t_pe, b->pblocks);
        else
            std::snprintf(buf, sizeof(buf), "; timed steps: phases %.4f ms, branches %.4f ms", t_ph, t_br);
        const std::string timed = std::string(buf) + pnote;
        if (t_br < t_ph && (t_pe < 0.f || t_br < t_pe)) {
            drop(b->graph, b->gexec);
            drop(g3, gx3);
            for (int p = 0; p < 2; p++) { b->graph[p] = g2[p]; b->gexec[p] = gx2[p]; }
            b->phases = false;
            b->plan = "branches: one graph branch per engine (chosen over the " + b->plan + ")" + timed;
        } else if (t_pe >= 0.f && t_pe < t_ph) {
            drop(b->graph, b->gexec);
            drop(g2, gx2);
            for (int p = 0; p < 2; p++) { b->graph[p] = g3[p]; b->gexec[p] = gx3[p]; }
            b->persistent = true;
            b->plan = "persistent: one cooperative launch per step over the " + b->plan.substr(8) + timed;
        } else {
            drop(g2, gx2);
            drop(g3, gx3);
            b->plan += timed;
        }
    }
    *out = b;
    return GF_OK;
}

int gf_batch_advance(gf_batch* b, uint64_t nsteps) {
    if (!b) return GF_EINVAL;
    GB_CU(cudaSetDevice(b->device));
    return batch_run(b, b->gexec, nsteps, nullptr, nullptr);
}

int gf_batch_synchronize(gf_batch* b) {
    if (!b) return GF_EINVAL;
    GB_CU(cudaStreamSynchronize(b->stream));
    return GF_OK;
}

void* gf_batch_stream(gf_batch* b) { return b ? (void*)b->stream : nullptr; }

int gf_batch_tuned_chunk(const gf_batch* b, int index) {
    if (!b || index < 0 || index >= (int)b->engs.size()) return -1;
    if (b->phases) return b->chunk[(size_t)index];
    return b->engs[(size_t)index]->el_chunk;
}

const char* gf_batch_plan(const gf_batch* b) { return b ? b->plan.c_str() : ""; }

const char* gf_batch_last_error(const gf_batch* b) { return b ? b->err.c_str() : g_create_err.c_str(); }

void gf_batch_destroy(gf_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (int p = 0; p < 2; p++) {
        if (b->gexec[p]) cudaGraphExecDestroy(b->gexec[p]);
        if (b->graph[p]) cudaGraphDestroy(b->graph[p]);
    }
    for (cudaEvent_t ev : b->join) if (ev) cudaEventDestroy(ev);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    for (cudaStream_t q : b->side) if (q) cudaStreamDestroy(q);
    for (cudaEvent_t ev : b->ev) if (ev) cudaEventDestroy(ev);
    if (b->dinst) cudaFree(b->dinst);
    if (b->dbar) cudaFree(b->dbar);
    for (BatchItem* p : b->ditems) if (p) cudaFree(p);
    delete b;
}

}  // extern "C"

// ===========================================================================
// Discrete adjoint of the ferromagnetic RK4 step (gf_adjoint_*)
//
// The forward run starts from the engine's current m and external-field
// clock, keeps the state every `ck_every` steps, and records <m_x> of every
// step.  The backward run walks the blocks between checkpoints in reverse.
// Store layout (when the block's stage fields fit in device memory): it
// recomputes the block from its checkpoint once, keeping every step's stage
// states, fields and strains, then applies the reverse RK4 sweep of
// gf_adjoint.cuh step by step from those.  Recompute layout: it recomputes
// and keeps the block's step values only, and recomputes each step's four
// stages (demag of each stage by FFT) again right before its sweep.  Both
// layouts run the same kernels on the same values, so their gradients are
// identical bit for bit.
// ===========================================================================
struct gf_adjoint {
    gf_engine* eng = nullptr;
    int nw = 0, ck_every = 0, nmat = 0;
    uint64_t nsteps = 0;
    bool ran = false;
    // on a mixed-form engine the adjoint's fields are FP32 (R = float), the
    // step values carry compensation words, and the gradients, the <m_x>
    // trace and its cotangent stay FP64; every buffer below except abar,
    // wbar, trace and dldm holds elements of esz bytes
    bool f32 = false;
    size_t esz = sizeof(double);
    std::vector<void*> allocs;
    void* am = nullptr;              // AdjMatT<R> per material
    double* aij = nullptr;           // (nmat+1)^2 harmonic-mean exchange constants
    double* alpha = nullptr;         // per cell
    std::vector<double> wave;        // excitation samples (A/m, x)
    std::vector<double> hext;        // nsteps x 4 x 3 external field of the deck per stage
    // state of a step: m (0-2); with elastodynamics also u (3-5), v (6-8)
    // and the stiffness-damping force store fs (9-11); in FP32 also the
    // compensation words of m (12-14), u (15-17) and v (18-20)
    bool el = false;
    int ns = 3;                      // components stored per step
    int sidx[21] = {};               // their indices in X
    double* X[21] = {};              // step value
    double* Y[3][3] = {};            // stage states y2, y3, y4 (m)
    double* ACC[3] = {};
    double* HS[4][3] = {};           // effective field of each stage
    double* XJ[3] = {};              // stage-4 output of a recomputed step (discarded)
    double* XJC[3] = {};             // and its compensation words (FP32)
    // cotangents: m (0-2), u (3-5), v (6-8)
    double* LAM[9] = {}; double* LAMACC[9] = {}; double* U[9] = {};
    double* YBAR[3] = {}; double* HBAR[3] = {};   // ybar of m (u's and v's stay in registers)
    double* abar = nullptr; double* hacc = nullptr; double* wbar = nullptr;   // FP64: alpha gradient, per-cell Hbar_x sum, waveform gradient
    // elastodynamics: stage u, v (stages 2-4), RK accumulators, the stage
    // force, the stage strain (LLG field), the cotangents of the force, the
    // stage-1 force of this step (f0bar) and of fs (phi), the transposed
    // stencil's pass-1 output (27 n), Liao history and pending cotangents
    double* US[3][3] = {}; double* VS[3][3] = {};
    double* UACC[3] = {}; double* VACC[3] = {};
    double* FORCE[3] = {};
    double* STR[4][6] = {};
    double* STRBAR[6] = {};
    double* FBAR[3] = {}; double* F0BAR[3] = {}; double* PHI[3] = {}; double* PHINEW[3] = {};
    double* TO = nullptr;
    double* hist = nullptr;          // 4 slots x 12 planes (k_elastic_bc's layout)
    double* last = nullptr;          // 3 planes
    double* pend = nullptr;          // 4 slots x 3 components x 4 planes
    double* trace = nullptr;         // nsteps+1 (FP64)
    size_t trace_len = 0;
    double* dldm = nullptr;          // nsteps+1 (FP64)
    double* ck = nullptr;            // checkpoints, (nsteps/ck_every + 1) x ck_len
    double* xs = nullptr;            // step values of one block, ck_every x ns n (recompute layout)
    size_t xs_bytes = 0;
    // stage store of one block (store layout): per step m of the step value,
    // the stage states, the stage fields and the stage strains
    double* store = nullptr;
    size_t store_bytes = 0;
    int64_t store_limit = -1;        // -1 automatic, 0 never, > 0 at most this many bytes
    bool store_used = false;         // layout of the last backward run
    double* zero3 = nullptr;         // 3n zeros (demag field when magnetostatics is off)
    double* wide = nullptr;          // FP32: 3n FP64 values of the final m
    size_t ck_slots = 0;
    size_t ck_len = 0;               // ns n (+ 51 planes of Liao state with elastodynamics)
};

namespace {

// zeroed device buffer of `count` elements of `bytes` each, complete on
// return (host copies may follow at once)
int adj_alloc_b(gf_adjoint* a, double** p, size_t count, size_t bytes) {
    gf_engine* eng = a->eng;
    GF_CU(cudaMalloc(p, count * bytes));
    a->allocs.push_back(*p);
    GF_CU(cudaMemsetAsync(*p, 0, count * bytes, eng->stream));
    GF_CU(cudaStreamSynchronize(eng->stream));
    return GF_OK;
}
// field elements (esz bytes) and FP64 elements
int adj_alloc(gf_adjoint* a, double** p, size_t count) { return adj_alloc_b(a, p, count, a->esz); }
int adj_alloc_d(gf_adjoint* a, double** p, size_t count) { return adj_alloc_b(a, p, count, sizeof(double)); }

int adj_alloc3(gf_adjoint* a, double* f[3]) {
    for (int c = 0; c < 3; c++) GF_TRY(adj_alloc(a, &f[c], (size_t)a->eng->P.n));
    return GF_OK;
}

// `elems` field elements past `base`
double* adj_at(const gf_adjoint* a, double* base, size_t elems) {
    return reinterpret_cast<double*>(reinterpret_cast<char*>(base) + elems * a->esz);
}
void adj_free(gf_adjoint* a, double** p) {
    if (!*p) return;
    cudaFree(*p);
    a->allocs.erase(std::remove(a->allocs.begin(), a->allocs.end(), (void*)*p), a->allocs.end());
    *p = nullptr;
}

// typed views of the buffers
template <class R> R* rp(double* p) { return reinterpret_cast<R*>(p); }
template <class R> F3T<R> v3(double* const* p) { F3T<R> r; for (int c = 0; c < 3; c++) r.c[c] = rp<R>(p[c]); return r; }
template <class R> F3T<R> v3c(R* base, long n) { F3T<R> r; for (int c = 0; c < 3; c++) r.c[c] = base + (size_t)c * n; return r; }
template <class R> const DevMatT<R>* adj_mats(const gf_engine* eng) {
    if constexpr (is_mixed<R>::value) return eng->mats_f;
    else return eng->mats;
}
template <class R> StageIOT<R> adj_base_io(const gf_engine* eng) {
    if constexpr (is_mixed<R>::value) return eng->iof[0][0];
    else return eng->io[0][0];
}

// demag field of stage state y (3 x n, left in the FFT buffer), or zeros;
// FP32: the mixed engine's R2C / six-spectra / C2R path
template <class R>
int adj_demag(gf_adjoint* a, F3T<R> y, F3T<R>& hd) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    if (eng->demag_mode != 0) { hd = v3c<R>(rp<R>(a->zero3), P.n); return GF_OK; }
    cudaStream_t st = eng->stream;
    const long n21 = (long)P.nx * P.ny * (P.nz / 2 + 1);
    if constexpr (is_mixed<R>::value) {
        float* M3 = reinterpret_cast<float*>(eng->Mfft);
        cufftComplex* Mk = reinterpret_cast<cufftComplex*>(eng->Mk);
        GF_CU(launch(k_mag_source_f32, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, st, P, (const DevMatT<float>*)eng->mats_f,
                     (const uint8_t*)eng->mid, y, F3T<float>{}, F3T<float>{}, 0, M3, f3f(eng->Hstat), 0.f, 0.f, 0.f));
        GF_FFT(cufftExecR2C(eng->plan_r2c, M3, Mk));
        const float inv_vol_neg = (float)(-1. / (P.dx * P.dy * P.dz));
        GF_CU(launch(k_demag_mul_f32, dim3(blocks_for(n21, kThreads)), dim3(kThreads), 0, st, n21, inv_vol_neg,
                     (const cuComplex*)Mk, (const float*)eng->Nr, (cuComplex*)Mk));
        GF_FFT(cufftExecC2R(eng->plan_c2r, Mk, M3));
        hd = v3c<float>(M3, P.n);
    } else {
        GF_CU(launch(k_mag_source, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, st, P, (const DevMat*)eng->mats,
                     (const uint8_t*)eng->mid, y, F3{}, F3{}, 0, eng->Mfft, f3(eng->Hstat), 0., 0., 0.));
        GF_FFT(cufftExecD2Z(eng->plan_r2c, eng->Mfft, eng->Mk));
        GF_CU(launch(k_demag_mul, dim3(blocks_for(n21, kThreads)), dim3(kThreads), 0, st, n21, -P.dx * P.dy * P.dz,
                     (const cuDoubleComplex*)eng->Mk, (const cuDoubleComplex*)eng->Nk, (cuDoubleComplex*)eng->Mk));
        GF_FFT(cufftExecZ2D(eng->plan_c2r, eng->Mk, eng->Mfft));
        hd = v3c<double>(eng->Mfft, P.n);
    }
    return GF_OK;
}

// the transposed convolution of Hbar (the operator is symmetric: the same
// transform pair and spectra), result 3 x n in the FFT buffer
template <class R>
int adj_demag_T(gf_adjoint* a, const R*& out) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    cudaStream_t st = eng->stream;
    const unsigned bn = blocks_for(P.n, kThreads);
    const long n21 = (long)P.nx * P.ny * (P.nz / 2 + 1);
    R* M3 = reinterpret_cast<R*>(eng->Mfft);
    GF_CU(launch(k_adj_pack<R>, dim3(bn), dim3(kThreads), 0, st, P, v3<R>(a->HBAR), M3));
    if constexpr (is_mixed<R>::value) {
        cufftComplex* Mk = reinterpret_cast<cufftComplex*>(eng->Mk);
        GF_FFT(cufftExecR2C(eng->plan_r2c, M3, Mk));
        const float inv_vol_neg = (float)(-1. / (P.dx * P.dy * P.dz));
        GF_CU(launch(k_demag_mul_f32, dim3(blocks_for(n21, kThreads)), dim3(kThreads), 0, st, n21, inv_vol_neg,
                     (const cuComplex*)Mk, (const float*)eng->Nr, (cuComplex*)Mk));
        GF_FFT(cufftExecC2R(eng->plan_c2r, Mk, M3));
    } else {
        GF_FFT(cufftExecD2Z(eng->plan_r2c, eng->Mfft, eng->Mk));
        GF_CU(launch(k_demag_mul, dim3(blocks_for(n21, kThreads)), dim3(kThreads), 0, st, n21, -P.dx * P.dy * P.dz,
                     (const cuDoubleComplex*)eng->Mk, (const cuDoubleComplex*)eng->Nk, (cuDoubleComplex*)eng->Mk));
        GF_FFT(cufftExecZ2D(eng->plan_c2r, eng->Mk, eng->Mfft));
    }
    out = M3;
    return GF_OK;
}

template <class R>
V3<R> adj_hext(const gf_adjoint* a, uint64_t step, int s) {
    const double* h = &a->hext[(size_t)(step * 4 + s) * 3];
    const size_t seg = (size_t)((step * (uint64_t)a->nw) / a->nsteps);
    return mk3<R>(R(h[0] + a->wave[seg]), R(h[1]), R(h[2]));
}

// StageIOT over the adjoint's buffers for the engine's elastic kernels: stage
// m and u in, the force and the stage strain out; for k_elastic_rk the step
// value (x), the stage v, the accumulators and the next stage's u, v (FP32:
// the step value's compensation words, which the last stage updates in place)
template <class R>
StageIOT<R> adj_el_io(gf_adjoint* a, double* const* x, F3T<R> ym, F3T<R> yu, F3T<R> yv, int s, F3T<R> uout, F3T<R> vout) {
    gf_engine* eng = a->eng;
    StageIOT<R> io = adj_base_io<R>(eng);     // tables, drive and materials of the engine
    io.m_in = ym;
    io.u_in = yu; io.v_in = yv;
    io.u_x = v3<R>(x + 3); io.v_x = v3<R>(x + 6);
    io.u_acc = v3<R>(a->UACC); io.v_acc = v3<R>(a->VACC);
    io.u_out = uout; io.v_out = vout;
    io.force = v3<R>(a->FORCE);
    io.force_store = v3<R>(x + 9);
    if (a->f32) { io.u_cmp = v3<R>(x + 15); io.v_cmp = v3<R>(x + 18); }
    for (int q = 0; q < 6; q++) { io.strain_c[q] = rp<R>(a->STR[s][q]); io.eps0_c[q] = nullptr; io.eig0_c[q] = nullptr;
                                  io.sg[q] = nullptr; io.pge[q] = nullptr; }
    return io;
}

// the engine's elastic tile (rk = 0) or RK update (rk = 1) of stage S on the
// adjoint's buffers; FP32 through the mixed translation unit, so that the
// adjoint's forward run is the mixed engine's own elastic discretisation
template <int S>
int adj_el_kernel(gf_adjoint* a, int rk, const StageIOT<double>& io) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    if (rk) {
        // the adjoint applies the Liao boundary itself, after the step
        Params Pa = P;
        Pa.el_bc_fused = 0;
        GF_CU(launch(k_elastic_rk<S, double>, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, eng->stream, Pa, io));
        return GF_OK;
    }
    ETileMaps tm;
    std::memset(&tm, 0, sizeof(tm));
    tm.err = eng->tma_err;
    const dim3 grid((P.nz + etile::TK - 1) / etile::TK, (P.ny + etile::TJ - 1) / etile::TJ,
                    (P.nx + eng->el_chunk - 1) / eng->el_chunk);
    if (eng->el_cubic)
        GF_CU(launch_tiled(k_elastic_tile<S, true, double>, grid, dim3(etile::NT), eng->el_smem, eng->stream, P, io,
                           eng->el_chunk, eng->el_nmat, tm));
    else
        GF_CU(launch_tiled(k_elastic_tile<S, false, double>, grid, dim3(etile::NT), eng->el_smem, eng->stream, P, io,
                           eng->el_chunk, eng->el_nmat, tm));
    return GF_OK;
}
template <class R>
int adj_el(gf_adjoint* a, int s, int rk, const StageIOT<R>& io) {
    if constexpr (is_mixed<R>::value) {
        return gf_mixed_adj_elastic(a->eng, s, rk, io);
    } else {
        if (s == 0) return adj_el_kernel<0>(a, rk, io);
        if (s == 1) return adj_el_kernel<1>(a, rk, io);
        if (s == 2) return adj_el_kernel<2>(a, rk, io);
        return adj_el_kernel<3>(a, rk, io);
    }
}

template <int S, class R>
cudaError_t adj_eval_launch(gf_adjoint* a, F3T<R> y, F3T<R> hd, V3<R> he, F3T<R> hs, F3T<R> xs_, F3T<R> xc, F3T<R> acc,
                            F3T<R> ynext, C6T<R> str) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    return launch(k_adj_eval<S, R>, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, eng->stream, P, (const uint8_t*)eng->mid,
                  (const AdjMatT<R>*)a->am, (const R*)rp<R>(a->aij), a->nmat, y, hd, (const R*)rp<R>(a->alpha), he, hs, xs_, xc,
                  acc, ynext, str);
}

// stages of step `step` from step value x: the effective fields go to HS,
// the stage states to Y (m) and US / VS (u, v), the stage strains to STR;
// stage 4 writes m to xout (compensation words to xcout in FP32; x itself in
// the forward run) and leaves the new u, v in UACC / VACC.  The elastic
// parts run the engine's own k_elastic_tile and k_elastic_rk (so the forward
// run is the engine's discretisation); k_elastic_rk of stage 1 stores the
// step's stage-1 force in x's fs.
template <class R>
int adj_stages(gf_adjoint* a, double* const* x, uint64_t step, F3T<R> xout, F3T<R> xcout) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    F3T<R> acc = v3<R>(a->ACC);
    F3T<R> xm = v3<R>(x);
    F3T<R> y = xm, yu{}, yv{};
    if (a->el) { yu = v3<R>(x + 3); yv = v3<R>(x + 6); }
    for (int s = 0; s < 4; s++) {
        F3T<R> hd;
        GF_TRY(adj_demag<R>(a, y, hd));
        C6T<R> str{};
        if (a->el) {
            const StageIOT<R> io = adj_el_io<R>(a, x, y, yu, yv, s, F3T<R>{}, F3T<R>{});
            GF_TRY(adj_el<R>(a, s, 0, io));
            if (P.elasto_on) for (int q = 0; q < 6; q++) str.c[q] = rp<R>(a->STR[s][q]);
        }
        const V3<R> he = adj_hext<R>(a, step, s);
        // stage 4 reads the step value from and writes the new one to xout:
        // x itself in the forward run (each thread reads its own cell before
        // writing it); a discarded buffer when a step is recomputed for the
        // reverse sweep, which needs only the stage fields
        F3T<R> ynext = (s < 3) ? v3<R>(a->Y[s]) : xout;
        F3T<R> xs_ = (s < 3) ? xm : xout;
        const F3T<R> hs = v3<R>(a->HS[s]);
        cudaError_t e;
        if (s == 0) e = adj_eval_launch<0, R>(a, y, hd, he, hs, xs_, F3T<R>{}, acc, ynext, str);
        else if (s == 1) e = adj_eval_launch<1, R>(a, y, hd, he, hs, xs_, F3T<R>{}, acc, ynext, str);
        else if (s == 2) e = adj_eval_launch<2, R>(a, y, hd, he, hs, xs_, F3T<R>{}, acc, ynext, str);
        else e = adj_eval_launch<3, R>(a, y, hd, he, hs, xs_, xcout, acc, ynext, str);
        GF_CU(e);
        if (a->el) {
            const F3T<R> uo = (s < 3) ? v3<R>(a->US[s]) : F3T<R>{}, vo = (s < 3) ? v3<R>(a->VS[s]) : F3T<R>{};
            const StageIOT<R> io = adj_el_io<R>(a, x, y, yu, yv, s, uo, vo);
            GF_TRY(adj_el<R>(a, s, 1, io));
            if (s < 3) { yu = v3<R>(a->US[s]); yv = v3<R>(a->VS[s]); }
        }
        if (s < 3) y = v3<R>(a->Y[s]);
    }
    return GF_OK;
}

// one forward step in place: m by k_adj_eval<3>, which reads x[c] before
// writing it in the same thread; then the Liao extrapolation of u(k = 0)
// and the new u, v from the accumulators
template <class R>
int adj_step_forward(gf_adjoint* a, double** x, uint64_t step) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    GF_TRY(adj_stages<R>(a, x, step, v3<R>(x), a->f32 ? v3<R>(x + 12) : F3T<R>{}));
    if (a->el) {
        const long plane = (long)P.nx * P.ny;
        GF_CU(launch(k_adj_liao<R>, dim3(blocks_for(plane, kThreads)), dim3(kThreads), 0, eng->stream, P, v3<R>(x + 3),
                     v3<R>(a->UACC), a->f32 ? v3<R>(x + 15) : F3T<R>{}, rp<R>(a->hist), rp<R>(a->last), (unsigned long long)step));
        // the new u, v are the accumulators: exchange the buffers
        for (int c = 0; c < 3; c++) { std::swap(x[3 + c], a->UACC[c]); std::swap(x[6 + c], a->VACC[c]); }
    }
    return GF_OK;
}

// FP64 sum of n field elements at `in` into p3 (three deterministic passes)
int adj_sum(gf_adjoint* a, const double* in, double*& p3) {
    gf_engine* eng = a->eng;
    cudaStream_t st = eng->stream;
    double* p1 = eng->scratch + eng->scratch_main;
    double* p2 = p1 + 8192;
    p3 = p2 + 64;
    if (a->f32) GF_CU(launch(k_sum_stride_f, dim3(32), dim3(256), 0, st, reinterpret_cast<const float*>(in), (long)eng->P.n, p1, 8192L));
    else GF_CU(launch(k_sum_stride, dim3(32), dim3(256), 0, st, in, (long)eng->P.n, p1, 8192L));
    GF_CU(launch(k_sum_stride, dim3(1), dim3(64), 0, st, (const double*)p1, 8192L, p2, 64L));
    GF_CU(launch(k_sum_stride, dim3(1), dim3(1), 0, st, (const double*)p2, 64L, p3, 1L));
    return GF_OK;
}

int adj_mean_x(gf_adjoint* a, const double* x0, long slot) {
    gf_engine* eng = a->eng;
    double* p3 = nullptr;
    GF_TRY(adj_sum(a, x0, p3));
    GF_CU(launch(k_adj_store_slot, dim3(1), dim3(1), 0, eng->stream, a->trace, slot, (const double*)p3,
                 1. / (double)eng->deck.NFM));
    return GF_OK;
}

// the waveform gradient of segment seg: the deterministic sum over cells of
// the per-cell Hbar_x sums of its steps, then those sums cleared
int adj_wave_flush(gf_adjoint* a, long seg) {
    gf_engine* eng = a->eng;
    cudaStream_t st = eng->stream;
    double* p1 = eng->scratch + eng->scratch_main;
    double* p2 = p1 + 8192;
    double* p3 = p2 + 64;
    GF_CU(launch(k_sum_stride, dim3(32), dim3(256), 0, st, (const double*)a->hacc, (long)eng->P.n, p1, 8192L));
    GF_CU(launch(k_sum_stride, dim3(1), dim3(64), 0, st, (const double*)p1, 8192L, p2, 64L));
    GF_CU(launch(k_sum_stride, dim3(1), dim3(1), 0, st, (const double*)p2, 64L, p3, 1L));
    GF_CU(launch(k_adj_add_slot, dim3(1), dim3(1), 0, st, a->wbar, seg, (const double*)p3));
    GF_CU(cudaMemsetAsync(a->hacc, 0, sizeof(double) * eng->P.n, st));
    return GF_OK;
}

// the elastic increments' cotangents: lambda / 6 at stage 4, U after
template <int S, class R>
cudaError_t adj_el_vjp_launch(gf_adjoint* a) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    double* const* uk = (S == 3) ? a->LAM : a->U;
    const R us = (S == 3) ? R(1. / 6.) : R(1);
    return launch(k_adj_el_vjp<S, R>, dim3(blocks_for(P.n, kThreads)), dim3(kThreads), 0, eng->stream, P, (const uint8_t*)eng->mid,
                  adj_mats<R>(eng), v3<R>(uk + 3), v3<R>(uk + 6), us, v3<R>(a->FBAR), v3<R>(a->LAM + 6), v3<R>(a->LAMACC + 6),
                  v3<R>(a->U + 6), v3<R>(a->F0BAR), v3<R>(a->PHI), v3<R>(a->PHINEW));
}
// reverse sweep of step `step` (lambda = d loss / d x_{step+1} in LAM on entry,
// d loss / d x_step on exit; with elastodynamics also phi = d loss / d fs);
// x is the step value x_step
// (recompute: the step's stages are formed here first; otherwise Y, HS and
// STR already hold them and only m of x is read)
template <class R>
int adj_step_backward(gf_adjoint* a, double* const* x, uint64_t step, bool recompute) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    cudaStream_t st = eng->stream;
    const unsigned bn = blocks_for(P.n, kThreads);
    const int ng = a->el ? 3 : 1;               // cotangent groups: m, u, v
    if (recompute) GF_TRY(adj_stages<R>(a, x, step, v3<R>(a->XJ), a->f32 ? v3<R>(a->XJC) : F3T<R>{}));
    if (a->el) {
        // the new u(k = 0) came from the Liao extrapolation, not the RK sum
        const long plane = (long)P.nx * P.ny;
        GF_CU(launch(k_adj_liao_T<R>, dim3(blocks_for(plane, kThreads)), dim3(kThreads), 0, st, P, v3<R>(a->LAM + 3),
                     rp<R>(a->pend), (unsigned long long)step));
        for (int c = 0; c < 3; c++) GF_CU(cudaMemsetAsync(a->F0BAR[c], 0, a->esz * P.n, st));
    }
    // the stage-4 cotangent u4 = lambda / 6 is read from lambda (scaled in
    // the kernels), and each group's RK combination runs in the kernel that
    // forms the group's final ybar (vjp + field_T [+ el_p1] for m, el_p2
    // for u, el_vjp for v), which writes lamacc (from lambda at stage 4)
    // and the next stage's u
    for (int s = 3; s >= 0; s--) {
        F3T<R> y = (s == 0) ? v3<R>(x) : v3<R>(a->Y[s - 1]);
        C6T<R> str{}, strbar{};
        if (a->el && P.elasto_on)
            for (int q = 0; q < 6; q++) { str.c[q] = rp<R>(a->STR[s][q]); strbar.c[q] = rp<R>(a->STRBAR[q]); }
        const F3T<R> um = (s == 3) ? v3<R>(a->LAM) : v3<R>(a->U);
        const R us = (s == 3) ? R(1. / 6.) : R(1);
        GF_CU(launch(k_adj_vjp<R>, dim3(bn), dim3(kThreads), 0, st, P, (const uint8_t*)eng->mid, (const AdjMatT<R>*)a->am, y,
                     v3<R>(a->HS[s]), um, us, (const R*)rp<R>(a->alpha), v3<R>(a->YBAR), v3<R>(a->HBAR), a->abar,
                     a->hacc, str, strbar));
        const R* Rk = nullptr;
        if (eng->demag_mode == 0) GF_TRY(adj_demag_T<R>(a, Rk));
        GF_CU(launch(k_adj_field_T<R>, dim3(bn), dim3(kThreads), 0, st, P, (const uint8_t*)eng->mid, (const AdjMatT<R>*)a->am,
                     (const R*)rp<R>(a->aij), a->nmat, v3<R>(a->HBAR), Rk, v3<R>(a->YBAR), a->el ? 0 : 1, s, v3<R>(a->LAM),
                     v3<R>(a->LAMACC), v3<R>(a->U)));
        if (a->el) {
            // elastic increments (and the v group's combination), then the
            // transposed stress and strain stencils (the m and u groups')
            cudaError_t e;
            if (s == 3) e = adj_el_vjp_launch<3, R>(a);
            else if (s == 2) e = adj_el_vjp_launch<2, R>(a);
            else if (s == 1) e = adj_el_vjp_launch<1, R>(a);
            else e = adj_el_vjp_launch<0, R>(a);
            GF_CU(e);
            GF_CU(launch(k_adj_el_p1<R>, dim3(bn), dim3(kThreads), 0, st, P, (const uint8_t*)eng->mid, adj_mats<R>(eng),
                         v3<R>(a->FBAR), strbar, y, v3<R>(a->YBAR), (int)P.elasto_back, rp<R>(a->TO), s, v3<R>(a->LAM),
                         v3<R>(a->LAMACC), v3<R>(a->U)));
            GF_CU(launch(k_adj_el_p2<R>, dim3(bn), dim3(kThreads), 0, st, P, (const uint8_t*)eng->mid, (const R*)rp<R>(a->TO),
                         s, v3<R>(a->LAM + 3), v3<R>(a->LAMACC + 3), v3<R>(a->U + 3)));
        }
    }
    for (int c = 0; c < 3 * ng; c++) std::swap(a->LAM[c], a->LAMACC[c]);
    if (a->el) {
        for (int c = 0; c < 3; c++) std::swap(a->PHI[c], a->PHINEW[c]);
        const long plane = (long)P.nx * P.ny;
        GF_CU(launch(k_adj_liao_pend<R>, dim3(blocks_for(plane, kThreads)), dim3(kThreads), 0, st, P, v3<R>(a->LAM + 3),
                     rp<R>(a->pend), (unsigned long long)step));
    }
    return GF_OK;
}

// precision dispatch
int adj_fwd(gf_adjoint* a, double** x, uint64_t step) {
    return a->f32 ? adj_step_forward<float>(a, x, step) : adj_step_forward<double>(a, x, step);
}
int adj_bwd(gf_adjoint* a, double* const* x, uint64_t step, bool recompute) {
    return a->f32 ? adj_step_backward<float>(a, x, step, recompute) : adj_step_backward<double>(a, x, step, recompute);
}

// elements of one step's slot in the stage store: m of the step value (3 n),
// the stage states y2..y4 (9 n), the four stage fields (12 n) and, with the
// magnetoelastic field, the four stage strains (24 n)
size_t adj_slot_len(const gf_adjoint* a) {
    return (size_t)((a->el && a->eng->P.elasto_on) ? 48 : 24) * (size_t)a->eng->P.n;
}

// points Y, HS (and STR) at a slot of the stage store while it lives, and
// puts the adjoint's own buffers back when it goes
struct AdjSlotView {
    gf_adjoint* a;
    double* Y[3][3];
    double* HS[4][3];
    double* STR[4][6];
    explicit AdjSlotView(gf_adjoint* a_) : a(a_) {
        std::memcpy(Y, a->Y, sizeof(Y)); std::memcpy(HS, a->HS, sizeof(HS)); std::memcpy(STR, a->STR, sizeof(STR));
    }
    ~AdjSlotView() {
        std::memcpy(a->Y, Y, sizeof(Y)); std::memcpy(a->HS, HS, sizeof(HS)); std::memcpy(a->STR, STR, sizeof(STR));
    }
    // slot `k` of the store; xm gets the slot's m of the step value
    void point(size_t k, double* xm[3]) {
        const size_t n = (size_t)a->eng->P.n;
        double* base = adj_at(a, a->store, k * adj_slot_len(a));
        size_t off = 0;
        for (int c = 0; c < 3; c++, off += n) xm[c] = adj_at(a, base, off);
        for (int s = 0; s < 3; s++)
            for (int c = 0; c < 3; c++, off += n) a->Y[s][c] = adj_at(a, base, off);
        for (int s = 0; s < 4; s++)
            for (int c = 0; c < 3; c++, off += n) a->HS[s][c] = adj_at(a, base, off);
        if (a->el && a->eng->P.elasto_on)
            for (int s = 0; s < 4; s++)
                for (int q = 0; q < 6; q++, off += n) a->STR[s][q] = adj_at(a, base, off);
    }
};

// the backward run's layout for blocks of kb steps: the stage store when it
// fits the limit and the device's free memory less a reserve of
// max(4 GiB, 1/16 of the device), else the step values (recompute layout)
int adj_prepare_backward(gf_adjoint* a, uint64_t kb) {
    gf_engine* eng = a->eng;
    const size_t need = (size_t)kb * adj_slot_len(a) * a->esz;
    a->store_used = false;
    if (a->store_limit != 0) {
        if (a->store && a->store_bytes >= need && (a->store_limit < 0 || need <= (size_t)a->store_limit)) {
            a->store_used = true;
        } else {
            adj_free(a, &a->store);
            a->store_bytes = 0;
            size_t fr = 0, tot = 0;
            GF_CU(cudaMemGetInfo(&fr, &tot));
            const size_t avail = fr + (a->xs ? a->xs_bytes : 0);
            const size_t reserve = std::max<size_t>((size_t)4 << 30, tot / 16);
            size_t budget = avail > reserve ? avail - reserve : 0;
            if (a->store_limit > 0) budget = std::min<size_t>(budget, (size_t)a->store_limit);
            if (need <= budget) {
                adj_free(a, &a->xs);
                a->xs_bytes = 0;
                if (cudaMalloc(&a->store, need) == cudaSuccess) {
                    a->allocs.push_back(a->store);
                    a->store_bytes = need;
                    a->store_used = true;
                } else {
                    (void)cudaGetLastError();
                    a->store = nullptr;
                }
            }
        }
    }
    if (!a->store_used) {
        adj_free(a, &a->store);
        a->store_bytes = 0;
        const size_t xneed = (size_t)kb * a->ns * (size_t)eng->P.n * a->esz;
        if (!a->xs || a->xs_bytes < xneed) {
            adj_free(a, &a->xs);
            a->xs_bytes = 0;
            GF_TRY(adj_alloc(a, &a->xs, (size_t)kb * a->ns * (size_t)eng->P.n));
            a->xs_bytes = xneed;
        }
    }
    return GF_OK;
}
int adj_inject(gf_adjoint* a, long slot, double inv_nfm) {
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    const dim3 g(blocks_for(P.n, kThreads));
    if (a->f32)
        GF_CU(launch(k_adj_inject<float>, g, dim3(kThreads), 0, eng->stream, P, (const uint8_t*)eng->mid,
                     (const AdjMatT<float>*)a->am, v3<float>(a->LAM), (const double*)a->dldm, slot, inv_nfm));
    else
        GF_CU(launch(k_adj_inject<double>, g, dim3(kThreads), 0, eng->stream, P, (const uint8_t*)eng->mid,
                     (const AdjMatT<double>*)a->am, v3<double>(a->LAM), (const double*)a->dldm, slot, inv_nfm));
    return GF_OK;
}

int adj_check(gf_adjoint* a) {
    if (!a || !a->eng) return GF_EINVAL;
    return GF_OK;
}

// the state x (ns arrays) to / from a contiguous slot, component-major; a
// checkpoint slot also holds the Liao history and last value
int adj_save(gf_adjoint* a, double* dst, bool liao) {
    gf_engine* eng = a->eng;
    const long n = eng->P.n, plane = (long)eng->P.nx * eng->P.ny;
    const size_t ez = a->esz;
    for (int q = 0; q < a->ns; q++)
        GF_CU(cudaMemcpyAsync(adj_at(a, dst, (size_t)q * n), a->X[a->sidx[q]], ez * n, cudaMemcpyDeviceToDevice, eng->stream));
    if (liao && a->el) {
        GF_CU(cudaMemcpyAsync(adj_at(a, dst, (size_t)a->ns * n), a->hist, ez * 48 * plane, cudaMemcpyDeviceToDevice, eng->stream));
        GF_CU(cudaMemcpyAsync(adj_at(a, dst, (size_t)a->ns * n + 48 * plane), a->last, ez * 3 * plane, cudaMemcpyDeviceToDevice,
                              eng->stream));
    }
    return GF_OK;
}
int adj_load(gf_adjoint* a, double* src, bool liao) {
    gf_engine* eng = a->eng;
    const long n = eng->P.n, plane = (long)eng->P.nx * eng->P.ny;
    const size_t ez = a->esz;
    for (int q = 0; q < a->ns; q++)
        GF_CU(cudaMemcpyAsync(a->X[a->sidx[q]], adj_at(a, src, (size_t)q * n), ez * n, cudaMemcpyDeviceToDevice, eng->stream));
    if (liao && a->el) {
        GF_CU(cudaMemcpyAsync(a->hist, adj_at(a, src, (size_t)a->ns * n), ez * 48 * plane, cudaMemcpyDeviceToDevice, eng->stream));
        GF_CU(cudaMemcpyAsync(a->last, adj_at(a, src, (size_t)a->ns * n + 48 * plane), ez * 3 * plane, cudaMemcpyDeviceToDevice,
                              eng->stream));
    }
    return GF_OK;
}

// material constants of the adjoint's dynamics in its real type
template <class R>
int adj_tables(gf_adjoint* a) {
    gf_engine* eng = a->eng;
    const Deck& d = eng->deck;
    std::vector<AdjMatT<R>> am(d.mats.size());
    for (size_t q = 0; q < d.mats.size(); q++) {
        const Material& m = d.mats[q];
        AdjMatT<R>& t = am[q];
        std::memset(&t, 0, sizeof(t));
        t.fm = m.fm ? 1u : 0u;
        if (m.fm) {
            t.gdt = R(m.gyro * d.dt); t.Ms = R(m.Ms); t.ex_coef = R(2. / kMu0 / m.Ms); t.Aex = R(m.Aex);
            t.K1c = R(m.K1 / kMu0 / m.Ms); t.K2c = R(m.K2 / kMu0 / m.Ms); t.aniso = (int)m.aniso_type;
            t.B1c = R(m.B1 / kMu0 / m.Ms); t.B2c = R(m.B2 / kMu0 / m.Ms);
        }
    }
    std::vector<R> aij((size_t)(a->nmat + 1) * (a->nmat + 1), R(0));
    for (int p = 0; p < a->nmat; p++)
        for (int q = 0; q < a->nmat; q++) {
            const double A1 = d.mats[p].Aex, A2 = d.mats[q].Aex;
            aij[(size_t)(p + 1) * (a->nmat + 1) + q + 1] = R((A1 + A2 != 0.) ? 2. * A1 * A2 / (A1 + A2) : 0.);
        }
    void* pm = nullptr;
    if (cudaMalloc(&pm, sizeof(AdjMatT<R>) * am.size()) != cudaSuccess) { eng->err = "cudaMalloc (adjoint tables)"; return GF_ENOMEM; }
    a->allocs.push_back(pm);
    a->am = pm;
    if (cudaMemcpy(a->am, am.data(), sizeof(AdjMatT<R>) * am.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        { eng->err = "cudaMemcpy (adjoint tables)"; return GF_ECUDA; }
    GF_TRY(adj_alloc(a, &a->aij, aij.size()));
    if (cudaMemcpy(a->aij, aij.data(), sizeof(R) * aij.size(), cudaMemcpyHostToDevice) != cudaSuccess)
        { eng->err = "cudaMemcpy (adjoint tables)"; return GF_ECUDA; }
    return GF_OK;
}

// per-cell damping from FP64 host values
int adj_upload_alpha(gf_adjoint* a, const double* al, size_t n) {
    gf_engine* eng = a->eng;
    if (a->f32) {
        std::vector<float> f(n);
        for (size_t c = 0; c < n; c++) f[c] = (float)al[c];
        GF_CU(cudaMemcpy(a->alpha, f.data(), sizeof(float) * n, cudaMemcpyHostToDevice));
    } else {
        GF_CU(cudaMemcpy(a->alpha, al, sizeof(double) * n, cudaMemcpyHostToDevice));
    }
    return GF_OK;
}

}  // namespace

extern "C" {

int gf_adjoint_create(gf_engine* e, int n_wave, int checkpoint_every, gf_adjoint** out) {
    GF_TRY(check(e));
    gf_engine* eng = e;
    if (!out || n_wave < 1 || checkpoint_every < 1) { eng->err = "gf_adjoint_create: need n_wave >= 1, checkpoint_every >= 1 and an output"; return GF_EINVAL; }
    *out = nullptr;
    const Deck& d = eng->deck;
    const Params& P = eng->P;
    if (!d.any_fm || d.any_afm || d.any_fe || d.em_dynamic)
        { eng->err = "the adjoint covers ferromagnetic LLG with magnetostatics and elastodynamics (no AFM, FE or Maxwell fields)"; return GF_EUNSUPPORTED; }
    if (d.elastodynamics) {
        if (d.abc_1D) { eng->err = "the adjoint covers the Liao boundary of the elastic run, not the Mur one (if_1D_ABC)"; return GF_EUNSUPPORTED; }
        if (d.strain_pulse) { eng->err = "the adjoint does not cover the elastic strain source"; return GF_EUNSUPPORTED; }
        if (P.ny < P.nz) { eng->err = "the adjoint needs ny >= nz (the reference's z-face neighbour rule for k = ny-1 is not transposed)"; return GF_EUNSUPPORTED; }
        if (P.nz < 5) { eng->err = "the adjoint's Liao boundary needs nz >= 5"; return GF_EUNSUPPORTED; }
        if (eng->es_eps[0] || eng->es_eig[0]) { eng->err = "the adjoint does not cover static strain inputs"; return GF_EUNSUPPORTED; }
    }
    if (P.rot) { eng->err = "the adjoint needs if_OrientRotate off"; return GF_EUNSUPPORTED; }
    if (eng->demag_mode > 0) { eng->err = "the adjoint covers the FFT magnetostatics (no demag factors / 1-D model)"; return GF_EUNSUPPORTED; }
    if (d.read_Hext_nonunif) { eng->err = "the adjoint does not cover a non-uniform external field"; return GF_EUNSUPPORTED; }
    for (const Material& m : d.mats)
        if (m.fm && m.iDMI != 0.) { eng->err = "the adjoint does not cover interfacial DMI"; return GF_EUNSUPPORTED; }
    GF_CU(cudaSetDevice(eng->device));
    gf_adjoint* a = new gf_adjoint();
    a->eng = eng; a->nw = n_wave; a->ck_every = checkpoint_every;
    a->nmat = (int)d.mats.size();
    a->f32 = eng->mixed;
    a->esz = a->f32 ? sizeof(float) : sizeof(double);
    a->wave.assign((size_t)n_wave, 0.);
    auto fail = [&](int rc) { gf_adjoint_destroy(a); return rc; };
    int rc = a->f32 ? adj_tables<float>(a) : adj_tables<double>(a);
    if (rc != GF_OK) return fail(rc);
    // per-cell damping, default the material's alpha
    const long n = P.n;
    if ((rc = adj_alloc(a, &a->alpha, (size_t)n)) != GF_OK) return fail(rc);
    {
        std::vector<double> al((size_t)n, 0.);
        for (long c = 0; c < n; c++) {
            const uint8_t id = d.material_cell[(size_t)c];
            if (id && d.mats[id - 1].fm) al[(size_t)c] = d.mats[id - 1].alpha;
        }
        if (adj_upload_alpha(a, al.data(), (size_t)n) != GF_OK) { eng->err = "cudaMemcpy (alpha)"; return fail(GF_ECUDA); }
    }
    a->el = d.elastodynamics;
    a->ns = 0;
    for (int q = 0; q < 3; q++) a->sidx[a->ns++] = q;
    if (a->el) for (int q = 3; q < 12; q++) a->sidx[a->ns++] = q;
    if (a->f32) {
        for (int q = 12; q < 15; q++) a->sidx[a->ns++] = q;
        if (a->el) for (int q = 15; q < 21; q++) a->sidx[a->ns++] = q;
    }
    double** bufs3[] = {a->X, a->ACC, a->XJ, a->LAM, a->LAMACC, a->U, a->YBAR, a->HBAR,
                        a->Y[0], a->Y[1], a->Y[2], a->HS[0], a->HS[1], a->HS[2], a->HS[3]};
    for (double** b : bufs3)
        if ((rc = adj_alloc3(a, b)) != GF_OK) return fail(rc);
    if (a->f32) {
        double** f3b[] = {a->X + 12, a->XJC};
        for (double** b : f3b)
            if ((rc = adj_alloc3(a, b)) != GF_OK) return fail(rc);
        if ((rc = adj_alloc_d(a, &a->wide, (size_t)3 * n)) != GF_OK) return fail(rc);
    }
    const long plane = (long)P.nx * P.ny;
    a->ck_len = (size_t)a->ns * n;
    if (a->el) {
        double** el3[] = {a->X + 3, a->X + 6, a->X + 9, a->LAM + 3, a->LAM + 6, a->LAMACC + 3, a->LAMACC + 6,
                          a->U + 3, a->U + 6, a->US[0], a->US[1], a->US[2],
                          a->VS[0], a->VS[1], a->VS[2], a->UACC, a->VACC, a->FORCE, a->FBAR, a->F0BAR, a->PHI, a->PHINEW};
        for (double** b : el3)
            if ((rc = adj_alloc3(a, b)) != GF_OK) return fail(rc);
        if (a->f32) {
            double** c3[] = {a->X + 15, a->X + 18};
            for (double** b : c3)
                if ((rc = adj_alloc3(a, b)) != GF_OK) return fail(rc);
        }
        for (int s_ = 0; s_ < 4; s_++)
            for (int q = 0; q < 6; q++)
                if ((rc = adj_alloc(a, &a->STR[s_][q], (size_t)n)) != GF_OK) return fail(rc);
        for (int q = 0; q < 6; q++)
            if ((rc = adj_alloc(a, &a->STRBAR[q], (size_t)n)) != GF_OK) return fail(rc);
        if ((rc = adj_alloc(a, &a->TO, (size_t)27 * n)) != GF_OK) return fail(rc);
        if ((rc = adj_alloc(a, &a->hist, (size_t)48 * plane)) != GF_OK) return fail(rc);
        if ((rc = adj_alloc(a, &a->last, (size_t)3 * plane)) != GF_OK) return fail(rc);
        if ((rc = adj_alloc(a, &a->pend, (size_t)48 * plane)) != GF_OK) return fail(rc);
        a->ck_len += (size_t)51 * plane;
    }
    if ((rc = adj_alloc_d(a, &a->abar, (size_t)n)) != GF_OK) return fail(rc);
    if ((rc = adj_alloc_d(a, &a->hacc, (size_t)n)) != GF_OK) return fail(rc);
    if ((rc = adj_alloc_d(a, &a->wbar, (size_t)n_wave)) != GF_OK) return fail(rc);
    if ((rc = adj_alloc(a, &a->zero3, (size_t)3 * n)) != GF_OK) return fail(rc);
    if (cudaStreamSynchronize(eng->stream) != cudaSuccess) { eng->err = "adjoint set-up"; return fail(GF_ECUDA); }
    *out = a;
    return GF_OK;
}

int gf_adjoint_set_alpha(gf_adjoint* a, const double* alpha, size_t count) {
    GF_TRY(adj_check(a));
    gf_engine* eng = a->eng;
    if (!alpha || count != (size_t)eng->P.n) { eng->err = "gf_adjoint_set_alpha: need nx*ny*nz values"; return GF_EINVAL; }
    return adj_upload_alpha(a, alpha, count);
}

int gf_adjoint_set_waveform(gf_adjoint* a, const double* w, size_t count) {
    GF_TRY(adj_check(a));
    gf_engine* eng = a->eng;
    if (!w || count != (size_t)a->nw) { eng->err = "gf_adjoint_set_waveform: need n_wave values"; return GF_EINVAL; }
    a->wave.assign(w, w + count);
    return GF_OK;
}

int gf_adjoint_forward(gf_adjoint* a, uint64_t nsteps, double* mx_trace) {
    GF_TRY(adj_check(a));
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    if (nsteps < 1 || !mx_trace) { eng->err = "gf_adjoint_forward: need nsteps >= 1 and a trace buffer of nsteps+1"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    cudaStream_t st = eng->stream;
    // external field of every stage from the engine's clock, which is restored
    const double t0 = eng->t_host;
    const long pH = eng->presc_H, pE = eng->presc_E;
    double hc[3], ec[3];
    std::memcpy(hc, eng->Hext_cur, sizeof(hc)); std::memcpy(ec, eng->Eext_cur, sizeof(ec));
    a->hext.assign((size_t)nsteps * 12, 0.);
    for (uint64_t k = 0; k < nsteps; k++) {
        StepDrive sd;
        step_drive(eng, sd);
        for (int s = 0; s < 4; s++)
            for (int c = 0; c < 3; c++) a->hext[(size_t)(k * 4 + s) * 3 + c] = sd.st[s].Hext[c];
    }
    eng->t_host = t0; eng->presc_H = pH; eng->presc_E = pE;
    std::memcpy(eng->Hext_cur, hc, sizeof(hc)); std::memcpy(eng->Eext_cur, ec, sizeof(ec));
    a->nsteps = nsteps;
    // checkpoints and traces sized for this run
    const size_t slots = (size_t)(nsteps / (uint64_t)a->ck_every) + 1;
    const long n = P.n;
    const size_t ez = a->esz;
    if (slots != a->ck_slots) {
        adj_free(a, &a->ck);
        a->ck_slots = 0;
    }
    if (!a->ck) {
        GF_TRY(adj_alloc(a, &a->ck, slots * a->ck_len));
        a->ck_slots = slots;
    }
    if (!a->trace || a->trace_len != (size_t)nsteps + 1) {
        // sized for this run's length (kept for further runs of the same length)
        adj_free(a, &a->trace);
        adj_free(a, &a->dldm);
        a->trace_len = 0;
        GF_TRY(adj_alloc_d(a, &a->trace, (size_t)nsteps + 1));
        GF_TRY(adj_alloc_d(a, &a->dldm, (size_t)nsteps + 1));
        a->trace_len = (size_t)nsteps + 1;
    }
    // initial state: the engine's current m (and u, v, force store, Liao
    // history: the engine's slot of its step e is the adjoint's slot of step
    // e - steps_done; in FP32 the compensation words)
    double* const* m0 = cur(eng, eng->m);
    for (int c = 0; c < 3; c++) GF_CU(cudaMemcpyAsync(a->X[c], m0[c], ez * n, cudaMemcpyDeviceToDevice, st));
    if (a->f32)
        for (int c = 0; c < 3; c++) GF_CU(cudaMemcpyAsync(a->X[12 + c], eng->m.C[c], ez * n, cudaMemcpyDeviceToDevice, st));
    if (a->el) {
        double* const* u0 = cur(eng, eng->u);
        double* const* v0 = cur(eng, eng->v);
        for (int c = 0; c < 3; c++) {
            GF_CU(cudaMemcpyAsync(a->X[3 + c], u0[c], ez * n, cudaMemcpyDeviceToDevice, st));
            GF_CU(cudaMemcpyAsync(a->X[6 + c], v0[c], ez * n, cudaMemcpyDeviceToDevice, st));
            GF_CU(cudaMemcpyAsync(a->X[9 + c], eng->force_store[c], ez * n, cudaMemcpyDeviceToDevice, st));
            if (a->f32) {
                GF_CU(cudaMemcpyAsync(a->X[15 + c], eng->u.C[c], ez * n, cudaMemcpyDeviceToDevice, st));
                GF_CU(cudaMemcpyAsync(a->X[18 + c], eng->v.C[c], ez * n, cudaMemcpyDeviceToDevice, st));
            }
        }
        const size_t plane = (size_t)P.nx * P.ny;
        for (int sl = 0; sl < 4; sl++)
            GF_CU(cudaMemcpyAsync(adj_at(a, a->hist, (size_t)sl * 12 * plane),
                                  reinterpret_cast<char*>(eng->liao_hist) + ((eng->steps_done + (uint64_t)sl) & 3ull) * 12 * plane * ez,
                                  ez * 12 * plane, cudaMemcpyDeviceToDevice, st));
        GF_CU(cudaMemcpyAsync(a->last, eng->liao_last, ez * 3 * plane, cudaMemcpyDeviceToDevice, st));
    }
    GF_TRY(adj_save(a, a->ck, true));
    GF_TRY(adj_mean_x(a, a->X[0], 0));
    for (uint64_t k = 0; k < nsteps; k++) {
        GF_TRY(adj_fwd(a, a->X, k));
        GF_TRY(adj_mean_x(a, a->X[0], (long)k + 1));
        if ((k + 1) % (uint64_t)a->ck_every == 0) {
            const size_t slot = (size_t)((k + 1) / (uint64_t)a->ck_every);
            GF_TRY(adj_save(a, adj_at(a, a->ck, slot * a->ck_len), true));
        }
    }
    GF_CU(cudaMemcpyAsync(mx_trace, a->trace, sizeof(double) * (nsteps + 1), cudaMemcpyDeviceToHost, st));
    // the engine's H_stat shares the FFT buffer the adjoint used
    GF_TRY(static_field_now(eng));
    GF_CU(cudaStreamSynchronize(st));
    a->ran = true;
    return GF_OK;
}

int gf_adjoint_backward(gf_adjoint* a, const double* dloss_dmx, double* grad_wave, double* grad_alpha) {
    GF_TRY(adj_check(a));
    gf_engine* eng = a->eng;
    const Params& P = eng->P;
    if (!a->ran) { eng->err = "gf_adjoint_backward: run gf_adjoint_forward first"; return GF_EINVAL; }
    if (!dloss_dmx || !grad_wave || !grad_alpha) { eng->err = "gf_adjoint_backward: null argument"; return GF_EINVAL; }
    GF_CU(cudaSetDevice(eng->device));
    cudaStream_t st = eng->stream;
    const long n = P.n;
    const size_t ez = a->esz;
    const uint64_t N = a->nsteps;
    const double inv_nfm = 1. / (double)eng->deck.NFM;
    GF_CU(cudaMemcpyAsync(a->dldm, dloss_dmx, sizeof(double) * (N + 1), cudaMemcpyHostToDevice, st));
    for (int c = 0; c < (a->el ? 9 : 3); c++) GF_CU(cudaMemsetAsync(a->LAM[c], 0, ez * n, st));
    if (a->el) {
        for (int c = 0; c < 3; c++) GF_CU(cudaMemsetAsync(a->PHI[c], 0, ez * n, st));
        GF_CU(cudaMemsetAsync(a->pend, 0, ez * 48 * (size_t)P.nx * P.ny, st));
    }
    GF_CU(cudaMemsetAsync(a->abar, 0, sizeof(double) * n, st));
    GF_CU(cudaMemsetAsync(a->wbar, 0, sizeof(double) * a->nw, st));
    GF_CU(cudaMemsetAsync(a->hacc, 0, sizeof(double) * n, st));
    long cur_seg = -1;                 // waveform segment whose Hbar_x sums hacc holds
    GF_TRY(adj_inject(a, (long)N, inv_nfm));
    const uint64_t K = (uint64_t)a->ck_every;
    const uint64_t nblocks = (N + K - 1) / K;
    GF_TRY(adj_prepare_backward(a, std::min<uint64_t>(K, N)));
    // the reverse sweep of step k from step value xp (m only in the store
    // layout), then the loss cotangent of step k
    auto sweep = [&](double* const* xp, uint64_t k, bool recompute) -> int {
        const long seg = (long)((k * (uint64_t)a->nw) / N);
        if (seg != cur_seg) {
            if (cur_seg >= 0) GF_TRY(adj_wave_flush(a, cur_seg));
            cur_seg = seg;
        }
        GF_TRY(adj_bwd(a, xp, k, recompute));
        return adj_inject(a, (long)k, inv_nfm);
    };
    for (uint64_t b = nblocks; b-- > 0;) {
        const uint64_t s0 = b * K, s1 = std::min(N, s0 + K);
        GF_TRY(adj_load(a, adj_at(a, a->ck, b * a->ck_len), true));
        if (a->store_used) {
            // recompute the block once, keeping every step's stages
            AdjSlotView view(a);
            double* xm[3];
            for (uint64_t k = s0; k < s1; k++) {
                view.point(k - s0, xm);
                for (int c = 0; c < 3; c++) GF_CU(cudaMemcpyAsync(xm[c], a->X[c], ez * n, cudaMemcpyDeviceToDevice, st));
                GF_TRY(adj_fwd(a, a->X, k));
            }
            for (uint64_t k = s1; k-- > s0;) {
                view.point(k - s0, xm);
                GF_TRY(sweep(xm, k, false));
            }
        } else {
            // recompute the block's step values x_s0 .. x_{s1-1}
            for (uint64_t k = s0; k < s1; k++) {
                GF_TRY(adj_save(a, adj_at(a, a->xs, (k - s0) * (size_t)a->ns * n), false));
                if (k + 1 < s1) GF_TRY(adj_fwd(a, a->X, k));
            }
            for (uint64_t k = s1; k-- > s0;) {
                double* xp[21] = {};
                for (int q = 0; q < a->ns; q++) xp[a->sidx[q]] = adj_at(a, a->xs, ((k - s0) * (size_t)a->ns + q) * n);
                GF_TRY(sweep(xp, k, true));
            }
        }
    }
    if (cur_seg >= 0) GF_TRY(adj_wave_flush(a, cur_seg));
    GF_CU(cudaMemcpyAsync(grad_wave, a->wbar, sizeof(double) * a->nw, cudaMemcpyDeviceToHost, st));
    GF_CU(cudaMemcpyAsync(grad_alpha, a->abar, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    GF_TRY(static_field_now(eng));
    GF_CU(cudaStreamSynchronize(st));
    return GF_OK;
}

int gf_adjoint_final_m(gf_adjoint* a, double* host_m, size_t count) {
    GF_TRY(adj_check(a));
    gf_engine* eng = a->eng;
    const long n = eng->P.n;
    if (!host_m || count != (size_t)(3 * n)) { eng->err = "gf_adjoint_final_m: need 3*nx*ny*nz values"; return GF_EINVAL; }
    if (!a->ran) { eng->err = "gf_adjoint_final_m: run gf_adjoint_forward first"; return GF_EINVAL; }
    // x of the last forward step: recompute from the last checkpoint
    const uint64_t K = (uint64_t)a->ck_every, N = a->nsteps;
    const uint64_t b = N / K;
    cudaStream_t st = eng->stream;
    GF_TRY(adj_load(a, adj_at(a, a->ck, b * a->ck_len), true));
    for (uint64_t k = b * K; k < N; k++) GF_TRY(adj_fwd(a, a->X, k));
    if (a->f32) {
        // FP64 values x + c of the compensated FP32 pairs
        for (int c = 0; c < 3; c++)
            GF_CU(launch(k_widen, dim3(blocks_for(n, kThreads)), dim3(kThreads), 0, st, (const float*)rp<float>(a->X[c]),
                         (const float*)rp<float>(a->X[12 + c]), n, a->wide + (size_t)c * n));
        GF_CU(cudaMemcpyAsync(host_m, a->wide, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st));
    } else {
        for (int c = 0; c < 3; c++)
            GF_CU(cudaMemcpyAsync(host_m + (size_t)c * n, a->X[c], sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    }
    GF_TRY(static_field_now(eng));
    GF_CU(cudaStreamSynchronize(st));
    return GF_OK;
}

int gf_adjoint_set_store_limit(gf_adjoint* a, int64_t bytes) {
    GF_TRY(adj_check(a));
    if (bytes < -1) { a->eng->err = "gf_adjoint_set_store_limit: need -1, 0 or a byte count"; return GF_EINVAL; }
    a->store_limit = bytes;
    return GF_OK;
}

int gf_adjoint_store_info(gf_adjoint* a, int* used, int64_t* bytes) {
    GF_TRY(adj_check(a));
    if (used) *used = a->store_used ? 1 : 0;
    if (bytes) *bytes = a->store_used ? (int64_t)a->store_bytes : (int64_t)a->xs_bytes;
    return GF_OK;
}

void gf_adjoint_destroy(gf_adjoint* a) {
    if (!a) return;
    if (a->eng && a->eng->stream) cudaStreamSynchronize(a->eng->stream);
    for (void* p : a->allocs) cudaFree(p);
    delete a;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free mean of a device array (gf_field_mean_noalloc).
//
// A deterministic three-pass strided sum (the k_sum_stride passes that
// gf_average also uses), with its partial sums in a file-scope device array
// instead of engine-owned scratch.  Pass 1 uses one partial per 1024 input
// elements (gf_average's pass 1 uses a fixed count of partials instead), so
// the result is deterministic for a given n but may differ from gf_average's
// in the last bits; the array bounds the input length; passes 2 and 3 reduce
// the partials to 64 values and then one.
// Every pass writes all the partials the next pass reads, so nothing in the
// array has to start at zero.  The array is shared by all calls on a device
// and keeps the last call's partials; calls that overlap on the GPU (two
// streams, two host threads) race on it.
// ---------------------------------------------------------------------------
namespace {
constexpr long kNoAllocPass1 = 65536;                       // pass-1 partials
constexpr long kNoAllocChunk = 1024;                        // elements per pass-1 partial
constexpr long kNoAllocMaxElems = kNoAllocPass1 * kNoAllocChunk;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocPass1 + 64 + 8];
constexpr int kMaxDevices = 64;
}  // namespace

extern "C" {

int gf_field_mean_noalloc(const double* dev_in, uint64_t n, double divisor, double* dev_out, void* stream) {
    auto fail = [](int code, const std::string& m) { g_create_err = m; return code; };
    if (!dev_in || !dev_out) return fail(GF_EINVAL, "gf_field_mean_noalloc: null device pointer");
    if (n == 0) return fail(GF_EINVAL, "gf_field_mean_noalloc: empty input");
    if (n > (uint64_t)kNoAllocMaxElems)
        return fail(GF_EINVAL, "gf_field_mean_noalloc: " + std::to_string(n) + " elements exceed the maximum of " +
                                   std::to_string(kNoAllocMaxElems) + " (fixed scratch of " +
                                   std::to_string(kNoAllocPass1) + " partial sums)");
    int dev = 0;
    cudaError_t ce = cudaGetDevice(&dev);
    if (ce != cudaSuccess) return fail(GF_ECUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
    if (dev < 0 || dev >= kMaxDevices) return fail(GF_ENODEV, "gf_field_mean_noalloc: device index out of range");
    // the device address of the file-scope array in the current device's
    // context (its host-side name is not a device address), looked up on
    // every call: a context that was reset and created again reloads the
    // module at another address
    void* addr = nullptr;
    ce = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (ce != cudaSuccess) return fail(GF_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(ce));
    double* scratch = static_cast<double*>(addr);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* p1 = scratch;
    double* p2 = scratch + kNoAllocPass1;
    const long T1 = (long)((n + kNoAllocChunk - 1) / kNoAllocChunk);
    // cudaLaunchKernel reports the error of its own launch; an error left
    // pending by the caller's earlier work stays for the caller to read
    const long nn = (long)n, c64 = 64L, c1 = 1L;
    const double* p1c = p1;
    const double* p2c = p2;
    void* a1[] = {(void*)&dev_in, (void*)&nn, (void*)&p1, (void*)&T1};
    void* a2[] = {(void*)&p1c, (void*)&T1, (void*)&p2, (void*)&c64};
    void* a3[] = {(void*)&p2c, (void*)&c64, (void*)&dev_out, (void*)&c1};
    void* a4[] = {(void*)&dev_out, (void*)&divisor};
    const void* ks = reinterpret_cast<const void*>(&k_sum_stride);
    ce = cudaLaunchKernel(ks, dim3(blocks_for(T1, 256)), dim3(256), a1, 0, st);
    if (ce == cudaSuccess) ce = cudaLaunchKernel(ks, dim3(1), dim3(64), a2, 0, st);
    if (ce == cudaSuccess) ce = cudaLaunchKernel(ks, dim3(1), dim3(1), a3, 0, st);
    if (ce == cudaSuccess) ce = cudaLaunchKernel(reinterpret_cast<const void*>(&k_scale), dim3(1), dim3(1), a4, 0, st);
    if (ce != cudaSuccess) return fail(GF_ECUDA, std::string("kernel launch: ") + cudaGetErrorString(ce));
    return GF_OK;
}


}  // extern "C"

#endif  // GF_MIXED_TU
