// Host-side description of a GO-Ferro run: the geometry block, the global
// switches of system_setting.in and the per-material constants of
// materials.in, with the same derived quantities the reference computes while
// reading them (read.cpp:4-215, global.cpp:14-441).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/goferro_b200.h"

namespace gf {

// One material (material.h:3-58) plus the derived constants the reference
// fills in read_materials / check_material / get_cijkl.
struct Material {
    double c11 = 0, c12 = 0, c44 = 0, density = 0;
    double mass_damping = 0, stiff_damping = 0;
    double cij[6][6] = {};                 // rotated stiffness (cijkl_glb)

    bool fm = false;
    double Ms = 0, gyro = 0, alpha = 0;
    unsigned aniso_type = 0;
    double K1 = 0, K2 = 0, Aex = 0, iDMI = 0;
    double lam100 = 0, lam111 = 0, B1 = 0, B2 = 0;

    bool afm = false;
    double Ms1 = 0, Ms2 = 0, gyro1 = 0, gyro2 = 0, alpha1 = 0, alpha2 = 0;
    double K1_1 = 0, K1_2 = 0, uaxis[3] = {0, 0, 0};
    double Aex1 = 0, Aex2 = 0, J_AFM = 0;
    double lam100_1 = 0, lam100_2 = 0, lam111_1 = 0, lam111_2 = 0;
    double B1_1 = 0, B1_2 = 0, B2_1 = 0, B2_2 = 0;

    bool spin_pump = false;
    double sh_angle = 0, sh_mixcond = 0, sh_difflen = 0;

    bool fe = false;
    double fe_mass = 0, fe_damping = 0;
    double a1 = 0, a11 = 0, a12 = 0, a111 = 0, a112 = 0, a123 = 0;
    double a1111 = 0, a1112 = 0, a1122 = 0, a1123 = 0;
    double G11 = 0, Q11 = 0, Q12 = 0, Q44 = 0;
    double f11 = 0, f12 = 0, f44 = 0, F11 = 0, F12 = 0, F44 = 0;
    double tv[8] = {};

    bool pec = false;
    double er = 1, cond = 0;
    double comp[3] = {}, wp[3] = {}, tau[3] = {};
};

struct Deck {
    // geometry block (read.cpp:217-237, geometry.cpp:3-44)
    long nx = 0, ny = 0, nz = 0;
    double dx = 0, dy = 0, dz = 0;
    bool per_x = true, per_y = true, per_z = true;
    bool read_struct = false;
    long nx_work = 0, ny_work = 0;
    long num_layer_unit = 0, num_periods = 1, id_firstlayer = 1, id_lastlayer_unit = 1;
    std::vector<unsigned> nz_layer_unit;
    std::vector<unsigned> nz_layer;        // expanded (set_geometry)
    long idxi = 0, idxf = 0, idyi = 0, idyf = 0, idzi = 0, idzf = 0;

    // globals (read.cpp:16-101)
    unsigned long long steps = 0;
    double dt = 0;
    unsigned num_materials = 0;
    std::vector<unsigned> material_layer_unit;
    bool orient_rotate = false;
    double Tg2c[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}, Tc2g[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    double theta_mag = 0, phi_mag = 0, px_init = 0, py_init = 0, pz_init = 0;
    bool read_Hext_nonunif = false;
    double Hext_stat[3] = {}, Hext_altr[3] = {}, H_altr_freq[3] = {};
    bool prescribe_H = false; long n_prescribe_H = 0;
    double Eext_stat[3] = {}, Eext_altr[3] = {}, E_altr_freq[3] = {};
    bool prescribe_E = false; long n_prescribe_E = 0;
    bool magnetostatics = false, mag_1D = false;
    bool demag_factor = false; double demag_fac[3] = {};
    bool elec_1D = false, elec_1D_comp = false;
    bool em_dynamic = false, planeEM = false;
    double planeEM_E[3] = {}, planeEM_freq[3] = {};
    bool em_fromP = false, em_fromM = false, em_back_P = false, em_back_M = false;
    long free_charge_nzi = 0, free_charge_nzf = 0; double free_charge = 0;
    double scale_elec = 0; unsigned elec_limit = 0; double elec_tol = 0;
    bool elastodynamics = false, elasto_back = false, elasto_on = false;
    bool strain_pulse = false; unsigned strain_type = 0; unsigned strain_z = 0;
    char strain_comp = 'x'; double sigma_gauss = 0, amp_gauss = 0; unsigned long strain_cycles = 0;
    bool elastostatic = false, elastostatic_1D = false, read_strain_ext = false, elastostatic_film = false;
    long strain_ext_nzi = 0, strain_ext_nzf = 0; double exx_ext = 0, eyy_ext = 0, exy_ext = 0;
    double scale_elasto = 0; unsigned elasto_limit = 0; double elasto_tol = 0;
    bool abc_1D = false, abc_elast_onlytop = false, abc_em_onlytop = false; double liao_w = 0;
    bool pec_xy = false, pec_z = false;
    bool flexo = false, spin_pumping = false;
    bool in_m = false, in_afm = false, in_Hstat = false, in_pq = false, in_Estat = false;
    bool in_em = false, in_Jp = false, in_uv = false, in_straint0 = false, in_eig0 = false, in_force = false;
    // output schedule of the time loop: switch and step interval of each of
    // the reference's text outputs (read.cpp; written by main.cpp:170-198 at
    // step 0 and main.cpp:486-705 after every step)
    struct Out { bool on = false; unsigned long long step = 0; };
    Out out_ave, out_m, out_magcell, out_AFMm, out_p, out_em, out_em_onecell;
    Out out_strain, out_Hstat, out_Estat, out_eig0, out_q, out_uv, out_force, out_emYee, out_Jp, out_Jishe;
    unsigned long long em_onecell_index = 0;
    bool jf_input = false;
    unsigned long jf_i0 = 0, jf_j0 = 0, jf_k0 = 0, jf_i1 = 0, jf_j1 = 0, jf_k1 = 0;
    unsigned jf_type = 0; char jf_comp = 'x'; double jf_amp = 0, jf_freq = 0, jf_sigma = 0; unsigned long jf_cycles = 0;
    bool prescribed_m = false; double precess_angle = 0, precess_freq = 0;

    std::vector<Material> mats;

    // derived (global.cpp:85-118)
    bool any_fm = false, any_fe = false, any_afm = false, any_pec = false;
    bool periodic_all = false;
    std::vector<uint8_t> material_cell;    // n cells, 0 = vacuum
    uint64_t NFM = 0, NFE = 0, NAFM = 0;

    // prescribed tables (Hext.in / Eext.in)
    std::vector<double> tH, Hx, Hy, Hz, tE, Ex, Ey, Ez;

    long n() const { return nx * ny * nz; }
};

// Fill a Deck from the host's parsed values (gf_create): the same fields
// and derived quantities read_deck produces from a deck directory, with no
// restart files.  Returns an empty string on success, else a message.
std::string deck_from_params(const gf_run_params& run, const gf_material_params* mats, int nmat,
                             const uint32_t* material_cell, Deck& d);

// Parse a deck directory.  Returns an empty string on success, else a
// message.  Restart files are not read here (the engine reads them with
// read_restart_vec3 / read_yee below).
std::string read_deck(const std::string& dir, Deck& d);

// "i j k a b c" (1-based) restart file with dims (nx, ny, nz) into three
// arrays (inoutput.cpp:11-27 layout).  Missing file leaves the arrays as
// they are (the reference skips a missing file).  `ncomp` values per line.
std::string read_restart(const std::string& path, long nx, long ny, long nz, int ncomp,
                         std::vector<double>* comps);

}  // namespace gf
