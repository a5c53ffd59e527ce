// The method-level binding a maintainer adds to GO-Ferro's C++ host to keep
// main.cpp and the four system classes' call sequence unchanged while the
// engine does the work (the replacement bodies of the classes' public
// methods: magnetic_system.h:158-211, ferroelectric_system.h:95-132,
// elastic_system.h:172-225, EMdynamic_system.h:131-180).
//
// Each get_d*_RK{s} opens stage s (gf_stage_begin), each update_*_RK{s} and
// the stage-4 update_* commit it (gf_stage_commit): the first commit of a
// stage runs the fused stage of every active physics, the others return at
// once.  The set-up keeps the reference's readers and hands their values to
// gf_create; static solves, averages and device copies map onto their ABI
// calls.
//
// tests/test_abi_consumer.py compiles this file against the reference's own
// headers (syntax and types: every replaced method must exist there with
// this signature); it is not linked into the engine or the tests.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "EMdynamic_system.h"
#include "elastic_system.h"
#include "ferroelectric_system.h"
#include "magnetic_system.h"
#include "goferro_b200.h"

gf_engine* g_engine = nullptr;    // created after the reference's set-up readers

namespace {
void check(int rc, const char* what) {
    if (rc != GF_OK) {
        std::fprintf(stderr, "%s: %s\n", what, gf_last_error(g_engine));
        std::abort();
    }
}
void begin(int s) { check(gf_stage_begin(g_engine, s), "gf_stage_begin"); }
void commit(int s) { check(gf_stage_commit(g_engine, s), "gf_stage_commit"); }

// one component-major field from the engine into three matrix3d arrays
void download3(int field, matrix3d<double>& x, matrix3d<double>& y, matrix3d<double>& z) {
    const size_t n = (size_t)x.dim;
    std::vector<double> buf(3 * n);
    check(gf_download(g_engine, field, buf.data(), buf.size()), "gf_download");
    for (size_t i = 0; i < n; i++) {
        x.matrix[i] = buf[i];
        y.matrix[i] = buf[n + i];
        z.matrix[i] = buf[2 * n + i];
    }
}
}  // namespace

// ---- magnetic_system --------------------------------------------------------
void magnetic_system::get_dm_RK1() { begin(1); }
void magnetic_system::get_dm_RK2() { begin(2); }
void magnetic_system::get_dm_RK3() { begin(3); }
void magnetic_system::get_dm_RK4() { begin(4); }
void magnetic_system::update_m_RK1() { commit(1); }
void magnetic_system::update_m_RK2() { commit(2); }
void magnetic_system::update_m_RK3() { commit(3); }
void magnetic_system::update_m() { commit(4); }
void magnetic_system::get_dm_AFM_RK1() { begin(1); }
void magnetic_system::get_dm_AFM_RK2() { begin(2); }
void magnetic_system::get_dm_AFM_RK3() { begin(3); }
void magnetic_system::get_dm_AFM_RK4() { begin(4); }
void magnetic_system::update_m_AFM_RK1() { commit(1); }
void magnetic_system::update_m_AFM_RK2() { commit(2); }
void magnetic_system::update_m_AFM_RK3() { commit(3); }
void magnetic_system::update_m_AFM() { commit(4); }
void magnetic_system::get_H_static() { check(gf_static_solve(g_engine, GF_STATIC_MAGNETIC), "gf_static_solve"); }
void magnetic_system::get_averagem() {
    double m[3];
    check(gf_average(g_engine, GF_OBS_M, m), "gf_average");
    mx_ave = m[0]; my_ave = m[1]; mz_ave = m[2];
}
void magnetic_system::copym_from_device() { download3(GF_FIELD_M, mx_glb, my_glb, mz_glb); }

// ---- ferroelectric_system ---------------------------------------------------
void ferroelectric_system::get_dq_RK1() { begin(1); }
void ferroelectric_system::get_dq_RK2() { begin(2); }
void ferroelectric_system::get_dq_RK3() { begin(3); }
void ferroelectric_system::get_dq_RK4() { begin(4); }
void ferroelectric_system::get_dp_RK1() { begin(1); }
void ferroelectric_system::get_dp_RK2() { begin(2); }
void ferroelectric_system::get_dp_RK3() { begin(3); }
void ferroelectric_system::get_dp_RK4() { begin(4); }
void ferroelectric_system::update_q_RK1() { commit(1); }
void ferroelectric_system::update_q_RK2() { commit(2); }
void ferroelectric_system::update_q_RK3() { commit(3); }
void ferroelectric_system::update_q() { commit(4); }
void ferroelectric_system::update_p_RK1() { commit(1); }
void ferroelectric_system::update_p_RK2() { commit(2); }
void ferroelectric_system::update_p_RK3() { commit(3); }
void ferroelectric_system::update_p() { commit(4); }
void ferroelectric_system::get_E_static() { check(gf_static_solve(g_engine, GF_STATIC_ELECTRIC), "gf_static_solve"); }
void ferroelectric_system::get_averagep() {
    double p[3];
    check(gf_average(g_engine, GF_OBS_P, p), "gf_average");
    px_ave = p[0]; py_ave = p[1]; pz_ave = p[2];
}
void ferroelectric_system::copyp_from_device() { download3(GF_FIELD_P, px_glb, py_glb, pz_glb); }

// ---- elastic_system -----------------------------------------------------------
void elastic_system::get_dv_RK1() { begin(1); }
void elastic_system::get_dv_RK2() { begin(2); }
void elastic_system::get_dv_RK3() { begin(3); }
void elastic_system::get_dv_RK4() { begin(4); }
void elastic_system::get_du_RK1() { begin(1); }
void elastic_system::get_du_RK2() { begin(2); }
void elastic_system::get_du_RK3() { begin(3); }
void elastic_system::get_du_RK4() { begin(4); }
void elastic_system::update_v_RK1() { commit(1); }
void elastic_system::update_u_RK1() { commit(1); }
void elastic_system::update_v_RK2() { commit(2); }
void elastic_system::update_u_RK2() { commit(2); }
void elastic_system::update_v_RK3() { commit(3); }
void elastic_system::update_u_RK3() { commit(3); }
void elastic_system::update_v() { commit(4); }
void elastic_system::update_u() { commit(4); }
void elastic_system::copy_uandv_from_device() {
    download3(GF_FIELD_U, Dux_glb, Duy_glb, Duz_glb);
    download3(GF_FIELD_V, vx_glb, vy_glb, vz_glb);
}

// ---- EMdynamic_system -------------------------------------------------------
void EMdynamic_system::get_dE_RK1() { begin(1); }
void EMdynamic_system::get_dE_RK2() { begin(2); }
void EMdynamic_system::get_dE_RK3() { begin(3); }
void EMdynamic_system::get_dE_RK4() { begin(4); }
void EMdynamic_system::get_dH_RK1() { begin(1); }
void EMdynamic_system::get_dH_RK2() { begin(2); }
void EMdynamic_system::get_dH_RK3() { begin(3); }
void EMdynamic_system::get_dH_RK4() { begin(4); }
void EMdynamic_system::update_DE_RK1() { commit(1); }
void EMdynamic_system::update_DE_RK2() { commit(2); }
void EMdynamic_system::update_DE_RK3() { commit(3); }
void EMdynamic_system::update_DE() { commit(4); }
void EMdynamic_system::update_DH_RK1() { commit(1); }
void EMdynamic_system::update_DH_RK2() { commit(2); }
void EMdynamic_system::update_DH_RK3() { commit(3); }
void EMdynamic_system::update_DH() { commit(4); }
