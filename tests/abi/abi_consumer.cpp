// A C++ program that uses the engine only through include/goferro_b200.h and
// libgoferro_b200.so, as a host that keeps the reference's main loop would:
//
//   abi_consumer DECK_DIR MODE STEPS [I J K]
//
// MODE "advance": one gf_advance per step (the replacement of the whole
//   loop body, main.cpp:243-484).
// MODE "stages": the reference's per-system call sequence of one step
//   (main.cpp:252-296 and its repetition for RK2..RK4): every system's
//   get_d*_RK{s} calls gf_stage_begin(e, s), every update_*_RK{s} (update_*
//   for s = 4) calls gf_stage_commit(e, s); only the first commit of a stage
//   launches it.
//
// Prints one line per step (step 0 = the initial state): the step, <m>,
// <m_AFM1>, <m_AFM2>, <p>, <u>, and the cell-centred E and H at (I,J,K), in
// the oracle's trace columns, %.17e.
//
// Test infrastructure (tests/test_abi_consumer.py builds and runs it).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "goferro_b200.h"

namespace {

void die(gf_engine* e, const char* what) {
    std::fprintf(stderr, "%s: %s\n", what, gf_last_error(e));
    std::exit(1);
}

#define CALL(e, x) do { if ((x) != GF_OK) die(e, #x); } while (0)

void trace(gf_engine* e, const gf_info& info, unsigned long long step, const long long probe[3]) {
    double row[21] = {0};
    if (info.fm) CALL(e, gf_average(e, GF_OBS_M, row + 0));
    if (info.afm) {
        CALL(e, gf_average(e, GF_OBS_M_AFM1, row + 3));
        CALL(e, gf_average(e, GF_OBS_M_AFM2, row + 6));
    }
    if (info.fe) CALL(e, gf_average(e, GF_OBS_P, row + 9));
    if (info.elastic) CALL(e, gf_average(e, GF_OBS_U, row + 12));
    if (info.em) CALL(e, gf_probe_em(e, probe[0], probe[1], probe[2], row + 15, row + 18));
    std::printf("%llu", step);
    for (double v : row) std::printf(" %.17e", v);
    std::printf("\n");
}

// The per-system methods of one RK stage in main.cpp's order; each system
// that is active calls the engine the way its replaced method would.
void stage_calls(gf_engine* e, const gf_info& info, int s) {
    // elastic_system::get_dv_RK{s}, get_du_RK{s}
    if (info.elastic) { CALL(e, gf_stage_begin(e, s)); CALL(e, gf_stage_begin(e, s)); }
    // magnetic_system::get_dm_RK{s} / get_dm_AFM_RK{s}
    if (info.fm) CALL(e, gf_stage_begin(e, s));
    if (info.afm) CALL(e, gf_stage_begin(e, s));
    // ferroelectric_system::get_dq_RK{s}, get_dp_RK{s}
    if (info.fe) { CALL(e, gf_stage_begin(e, s)); CALL(e, gf_stage_begin(e, s)); }
    // EMdynamic_system::get_dE_RK{s}, get_dH_RK{s}
    if (info.em) { CALL(e, gf_stage_begin(e, s)); CALL(e, gf_stage_begin(e, s)); }
    // the update_*_RK{s} methods, each system in turn
    if (info.elastic) { CALL(e, gf_stage_commit(e, s)); CALL(e, gf_stage_commit(e, s)); }
    if (info.fm) CALL(e, gf_stage_commit(e, s));
    if (info.afm) CALL(e, gf_stage_commit(e, s));
    if (info.fe) { CALL(e, gf_stage_commit(e, s)); CALL(e, gf_stage_commit(e, s)); }
    if (info.em) { CALL(e, gf_stage_commit(e, s)); CALL(e, gf_stage_commit(e, s)); }
    // a run with no system active in this stage still commits it
    CALL(e, gf_stage_commit(e, s));
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 4 && argc != 7) {
        std::fprintf(stderr, "usage: %s DECK_DIR advance|stages STEPS [I J K]\n", argv[0]);
        return 2;
    }
    const bool stages = std::strcmp(argv[2], "stages") == 0;
    if (!stages && std::strcmp(argv[2], "advance") != 0) {
        std::fprintf(stderr, "mode must be advance or stages\n");
        return 2;
    }
    const unsigned long long steps = std::strtoull(argv[3], nullptr, 10);
    long long probe[3] = {0, 0, 0};
    if (argc == 7)
        for (int a = 0; a < 3; a++) probe[a] = std::atoll(argv[4 + a]);

    gf_engine* e = nullptr;
    if (gf_create_from_deck(argv[1], 0, &e) != GF_OK) die(nullptr, "gf_create_from_deck");
    gf_info info;
    CALL(e, gf_get_info(e, &info));
    trace(e, info, 0, probe);
    for (unsigned long long n = 1; n <= steps; n++) {
        if (stages) {
            for (int s = 1; s <= 4; s++) stage_calls(e, info, s);
        } else {
            CALL(e, gf_advance(e, 1));
        }
        trace(e, info, n, probe);
    }
    CALL(e, gf_check_finite(e));
    gf_destroy(e);
    return 0;
}
