// GO-Ferro input-deck reader.  The decks are positional text files; this
// reads them field by field in the order the reference does
// (read.cpp:4-111 system_setting.in, read.cpp:113-215 materials.in,
// read.cpp:217-237 geometry block) and derives what set_geometry
// (geometry.cpp:3-44), set_global (global.cpp:14-320), check_material
// (global.cpp:322-363) and get_cijkl (global.cpp:365-441) derive.  Unlike
// the reference it reports a malformed or missing deck instead of running
// on uninitialised values.
#include "gf_deck.h"

#include <cmath>
#include <fstream>
#include <sstream>

namespace gf {
namespace {

struct Reader {
    std::ifstream f;
    std::string err;
    std::string what;
    template <class T> Reader& get(T& v, const char* name) {
        if (!err.empty()) return *this;
        f >> v;
        if (f.fail()) err = std::string("cannot read '") + name + "' (" + what + ")";
        return *this;
    }
    Reader& flag(bool& v, const char* name) {
        if (!err.empty()) return *this;
        f >> std::boolalpha >> v;
        if (f.fail()) err = std::string("cannot read boolean '") + name + "' (" + what + ")";
        return *this;
    }
    void eol() { if (err.empty()) f.ignore(1000, '\n'); }
};

void expand_layers(Deck& d) {
    // geometry.cpp:3-44 — repeat the unit layers [id_firstlayer,
    // id_lastlayer_unit] num_periods times
    long num_unit = d.id_lastlayer_unit - d.id_firstlayer + 1;
    long id_last = d.id_firstlayer - 1 + d.num_periods * num_unit;
    long num_layer = d.num_layer_unit + (d.num_periods - 1) * num_unit;
    d.nz_layer.assign(num_layer > 0 ? num_layer : 0, 0);
    std::vector<unsigned> mat_layer(d.nz_layer.size(), 0);
    long j = d.id_firstlayer;
    for (long i = 0; i < num_layer; i++) {
        long src;
        if (i < d.id_firstlayer - 1) src = i;
        else if (i > id_last - 1) src = i - num_layer + d.num_layer_unit;
        else { src = j - 1; j = j + 1; if (j > d.id_lastlayer_unit) j = d.id_firstlayer; }
        d.nz_layer[i] = d.nz_layer_unit[src];
        mat_layer[i] = d.material_layer_unit[src];
    }
    long nz_work = 0;
    for (unsigned v : d.nz_layer) nz_work += v;
    d.idxi = (d.nx - d.nx_work) / 2;
    d.idxf = d.idxi + d.nx_work - 1;
    d.idyi = (d.ny - d.ny_work) / 2;
    d.idyf = d.idyi + d.ny_work - 1;
    d.idzi = 0;
    d.idzf = nz_work - 1;
    // material per cell (global.cpp:65-79)
    d.material_cell.assign((size_t)d.n(), 0);
    long zf = -1;
    for (size_t l = 0; l < d.nz_layer.size(); l++) {
        long zi = zf + 1;
        zf = zi + d.nz_layer[l] - 1;
        for (long i = d.idxi; i <= d.idxf; i++)
            for (long jj = d.idyi; jj <= d.idyf; jj++)
                for (long k = zi; k <= zf; k++)
                    d.material_cell[(size_t)((i * d.ny + jj) * d.nz + k)] = (uint8_t)mat_layer[l];
    }
}

void derive_material(Material& m, const double Tc2g[3][3]) {
    // read.cpp:141-142,162-165,184-198
    m.B1 = -3. / 2. * m.lam100 * (m.c11 - m.c12);
    m.B2 = -3. * m.lam111 * m.c44;
    m.B1_1 = -3. / 2. * m.lam100_1 * (m.c11 - m.c12);
    m.B1_2 = -3. / 2. * m.lam100_2 * (m.c11 - m.c12);
    m.B2_1 = -3. * m.lam111_1 * m.c44;
    m.B2_2 = -3. * m.lam111_2 * m.c44;
    m.F11 = ((m.c11 + m.c12) * m.f11 - 2. * m.c12 * m.f12) / (m.c11 + 2. * m.c12) / (m.c11 - m.c12);
    m.F12 = (m.c11 * m.f12 - m.c12 * m.f11) / (m.c11 + 2. * m.c12) / (m.c11 - m.c12);
    m.F44 = m.f44 / m.c44;
    const double c11 = m.c11, c12 = m.c12, c44 = m.c44, Q11 = m.Q11, Q12 = m.Q12, Q44 = m.Q44;
    const double F11 = m.F11, F12 = m.F12, F44 = m.F44;
    m.tv[0] = 2. * (c11 * Q11 + 2. * c12 * Q12);
    m.tv[1] = 2. * (c11 * Q12 + c12 * Q11 + c12 * Q12);
    m.tv[2] = 4. * c44 * Q44;
    m.tv[3] = 2. * (c11 * (Q11 * F11 + 2. * Q12 * F12) + 2. * c12 * (Q11 * F12 + Q12 * F11 + Q12 * F12));
    m.tv[4] = 2. * (c11 * (Q11 * F12 + Q12 * F11 + Q12 * F12) + c12 * (Q11 * F11 + Q11 * F12 + Q12 * F11 + 3. * Q12 * F12));
    m.tv[5] = 2. * c44 * Q44 * F44;
    m.tv[6] = c11 * (F11 * F11 + 2. * F12 * F12) + 2. * c12 * (F12 * F12 + 2. * F11 * F12);
    m.tv[7] = c44 * F44 * F44;

    // check_material (global.cpp:322-363): zero the constants of absent
    // orders; the Drude weights are renormalised one after another, each
    // with the already-updated values before it
    if (!m.fm) { m.Ms = m.gyro = m.alpha = 0; m.aniso_type = 0; m.K1 = m.K2 = m.Aex = m.iDMI = 0;
                 m.lam100 = m.lam111 = m.B1 = m.B2 = 0; }
    if (!m.afm) { m.Ms1 = m.Ms2 = m.gyro1 = m.gyro2 = m.alpha1 = m.alpha2 = 0; m.K1_1 = m.K1_2 = 0;
                  m.Aex1 = m.Aex2 = m.J_AFM = 0; m.lam100_1 = m.lam100_2 = m.lam111_1 = m.lam111_2 = 0;
                  m.B1_1 = m.B1_2 = m.B2_1 = m.B2_2 = 0; }
    if (!m.fe) { m.fe_mass = m.fe_damping = 0; m.a1 = m.a11 = m.a12 = m.a111 = m.a112 = m.a123 = 0;
                 m.a1111 = m.a1112 = m.a1122 = m.a1123 = 0; m.G11 = m.Q11 = m.Q12 = m.Q44 = 0;
                 for (double& t : m.tv) t = 0; m.f11 = m.f12 = m.f44 = 0; m.F11 = m.F12 = m.F44 = 0; }
    m.comp[0] = m.comp[0] / (m.comp[0] + m.comp[1] + m.comp[2]);
    m.comp[1] = m.comp[1] / (m.comp[0] + m.comp[1] + m.comp[2]);
    m.comp[2] = m.comp[2] / (m.comp[0] + m.comp[1] + m.comp[2]);

    // get_cijkl: Voigt 6x6 -> 4th-rank tensor, rotate with Tc2g, back to Voigt
    static const int vw[6] = {0, 1, 2, 1, 0, 0}, vx[6] = {0, 1, 2, 2, 2, 1};
    double Ccrt[6][6] = {};
    Ccrt[0][0] = Ccrt[1][1] = Ccrt[2][2] = m.c11;
    Ccrt[0][1] = Ccrt[0][2] = Ccrt[1][2] = Ccrt[1][0] = Ccrt[2][0] = Ccrt[2][1] = m.c12;
    Ccrt[3][3] = Ccrt[4][4] = Ccrt[5][5] = m.c44;
    double C4[3][3][3][3] = {}, R4[3][3][3][3] = {};
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) {
            int w = vw[a], x = vx[a], y = vw[b], z = vx[b];
            C4[w][x][y][z] = C4[x][w][y][z] = C4[w][x][z][y] = C4[x][w][z][y] = Ccrt[a][b];
        }
    for (int w = 0; w < 3; w++) for (int x = 0; x < 3; x++) for (int y = 0; y < 3; y++) for (int z = 0; z < 3; z++)
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) for (int k = 0; k < 3; k++) for (int l = 0; l < 3; l++)
            R4[w][x][y][z] = R4[w][x][y][z] + Tc2g[w][i] * Tc2g[x][j] * Tc2g[y][k] * Tc2g[z][l] * C4[i][j][k][l];
    for (int a = 0; a < 6; a++)
        for (int b = 0; b < 6; b++) m.cij[a][b] = R4[vw[a]][vx[a]][vw[b]][vx[b]];
}

std::string read_materials(const std::string& dir, Deck& d) {
    Reader r;
    r.f.open(dir + "/materials.in");
    if (!r.f.is_open()) return "cannot open " + dir + "/materials.in";
    d.mats.assign(d.num_materials, Material());
    for (unsigned i = 0; i < d.num_materials; i++) {
        Material& m = d.mats[i];
        std::string title;
        std::getline(r.f, title);
        r.what = "materials.in, material " + std::to_string(i + 1);
        r.get(m.c11, "c11").get(m.c12, "c12").get(m.c44, "c44"); r.eol();
        r.get(m.density, "density"); r.eol();
        r.get(m.mass_damping, "elast_mass_damping").get(m.stiff_damping, "elast_stiff_damping"); r.eol();
        r.flag(m.fm, "if_FM"); r.eol();
        r.get(m.Ms, "Ms").get(m.gyro, "gyro").get(m.alpha, "FM_damping"); r.eol();
        r.get(m.aniso_type, "anisotropy_type"); r.eol();
        r.get(m.K1, "K1").get(m.K2, "K2"); r.eol();
        r.get(m.Aex, "Aex"); r.eol();
        r.get(m.iDMI, "iDMI"); r.eol();
        r.get(m.lam100, "lamda100").get(m.lam111, "lamda111"); r.eol();
        r.flag(m.afm, "if_AFM"); r.eol();
        r.get(m.Ms1, "Ms_AFM1").get(m.Ms2, "Ms_AFM2"); r.eol();
        r.get(m.gyro1, "gyro_AFM1").get(m.gyro2, "gyro_AFM2"); r.eol();
        r.get(m.alpha1, "damping_AFM1").get(m.alpha2, "damping_AFM2"); r.eol();
        r.get(m.K1_1, "K1_AFM1").get(m.K1_2, "K1_AFM2"); r.eol();
        r.get(m.uaxis[0], "uniaxis_x").get(m.uaxis[1], "uniaxis_y").get(m.uaxis[2], "uniaxis_z"); r.eol();
        {
            double norm = std::sqrt(m.uaxis[0] * m.uaxis[0] + m.uaxis[1] * m.uaxis[1] + m.uaxis[2] * m.uaxis[2]);
            m.uaxis[0] = m.uaxis[0] / norm; m.uaxis[1] = m.uaxis[1] / norm; m.uaxis[2] = m.uaxis[2] / norm;
        }
        r.get(m.Aex1, "Aex_AFM1").get(m.Aex2, "Aex_AFM2"); r.eol();
        r.get(m.J_AFM, "J_AFM"); r.eol();
        r.get(m.lam100_1, "lamda100_AFM1").get(m.lam100_2, "lamda100_AFM2"); r.eol();
        r.get(m.lam111_1, "lamda111_AFM1").get(m.lam111_2, "lamda111_AFM2"); r.eol();
        r.flag(m.spin_pump, "if_spin_pump"); r.eol();
        r.get(m.sh_angle, "spin_hall_angle").get(m.sh_mixcond, "spin_mix_cond").get(m.sh_difflen, "spin_diffus_length"); r.eol();
        r.flag(m.fe, "if_FE"); r.eol();
        r.get(m.fe_mass, "FE_mass").get(m.fe_damping, "FE_damping"); r.eol();
        r.get(m.a1, "a1"); r.eol();
        r.get(m.a11, "a11").get(m.a12, "a12"); r.eol();
        r.get(m.a111, "a111").get(m.a112, "a112").get(m.a123, "a123"); r.eol();
        r.get(m.a1111, "a1111").get(m.a1112, "a1112").get(m.a1122, "a1122").get(m.a1123, "a1123"); r.eol();
        r.get(m.G11, "G11"); r.eol();
        r.get(m.Q11, "Q11").get(m.Q12, "Q12").get(m.Q44, "Q44"); r.eol();
        r.get(m.f11, "f11").get(m.f12, "f12").get(m.f44, "f44"); r.eol();
        r.flag(m.pec, "if_PEC"); r.eol();
        r.get(m.er, "r_permittivity"); r.eol();
        r.get(m.cond, "conductivity"); r.eol();
        for (int p = 0; p < 3; p++) { r.get(m.comp[p], "comp_n").get(m.wp[p], "omega_plasma").get(m.tau[p], "tao_e"); r.eol(); }
        if (!r.err.empty()) return r.err;
        derive_material(m, d.Tc2g);
    }
    return "";
}

std::string read_table(const std::string& path, long n, std::vector<double>& t, std::vector<double>& x,
                       std::vector<double>& y, std::vector<double>& z) {
    t.assign(n, 0.); x.assign(n, 0.); y.assign(n, 0.); z.assign(n, 0.);
    std::ifstream f(path);
    if (!f.is_open()) return "";  // the reference leaves the table at whatever new[] gave; we keep zeros
    for (long i = 0; i < n; i++) f >> t[i] >> x[i] >> y[i] >> z[i];
    if (f.fail()) return "malformed table " + path;
    return "";
}

// counts and flags set_global derives from the materials and the cells
// (global.cpp:85-118), and the demag factors normalised to sum -1
// (global.cpp:271-275)
void finish_deck(Deck& d) {
    for (const Material& m : d.mats) {
        d.any_fm |= m.fm; d.any_fe |= m.fe; d.any_afm |= m.afm; d.any_pec |= m.pec;
    }
    d.NFM = d.NFE = d.NAFM = 0;
    for (uint8_t id : d.material_cell)
        if (id) { const Material& m = d.mats[id - 1]; d.NFM += m.fm; d.NFE += m.fe; d.NAFM += m.afm; }
    d.periodic_all = d.per_x && d.per_y && d.per_z;

    // demag factors normalised to sum -1 (global.cpp:271-275)
    {
        double norm = d.demag_fac[0] + d.demag_fac[1] + d.demag_fac[2];
        for (int i = 0; i < 3; i++) d.demag_fac[i] = d.demag_fac[i] / norm * -1.;
    }
}

}  // namespace

std::string read_deck(const std::string& dir, Deck& d) {
    Reader r;
    r.f.open(dir + "/system_setting.in");
    if (!r.f.is_open()) return "cannot open " + dir + "/system_setting.in";
    r.what = "system_setting.in geometry block";
    r.get(d.nx, "nx").get(d.ny, "ny").get(d.nz, "nz"); r.eol();
    r.get(d.dx, "dx").get(d.dy, "dy").get(d.dz, "dz"); r.eol();
    r.flag(d.per_x, "periodicX").flag(d.per_y, "periodicY").flag(d.per_z, "periodicZ"); r.eol();
    r.flag(d.read_struct, "if_read_struct"); r.eol();
    r.get(d.nx_work, "nx_work").get(d.ny_work, "ny_work"); r.eol();
    r.get(d.num_layer_unit, "num_layer_unit"); r.eol();
    r.get(d.num_periods, "num_periods").get(d.id_firstlayer, "id_firstlayer").get(d.id_lastlayer_unit, "id_lastlayer_unit"); r.eol();
    if (!r.err.empty()) return r.err;
    if (d.nx < 1 || d.ny < 1 || d.nz < 1) return "grid dimensions must be positive";
    if (d.num_layer_unit < 1 || d.num_layer_unit > 100000) return "bad num_layer_unit";
    d.nz_layer_unit.assign(d.num_layer_unit, 0);
    for (long i = 0; i < d.num_layer_unit; i++) r.get(d.nz_layer_unit[i], "nz of layer unit");
    if (!r.err.empty()) return r.err;
    r.f.close();

    // read_global skips the first 8 non-empty lines (read.cpp:10-15)
    r.f.clear();
    r.f.open(dir + "/system_setting.in");
    std::string line;
    for (int i = 0; i < 8;) {
        if (!std::getline(r.f, line)) return "system_setting.in: geometry block shorter than 8 non-empty lines";
        if (line.length() > 0) i = i + 1;
    }
    r.what = "system_setting.in";
    r.get(d.steps, "step"); r.eol();
    r.get(d.dt, "dt"); r.eol();
    r.get(d.num_materials, "num_materials"); r.eol();
    if (!r.err.empty()) return r.err;
    if (d.num_materials < 1 || d.num_materials > 255) return "num_materials must be 1..255";
    d.material_layer_unit.assign(d.num_layer_unit, 0);
    for (long i = 0; i < d.num_layer_unit; i++) r.get(d.material_layer_unit[i], "material id of layer unit");
    r.eol();
    r.flag(d.orient_rotate, "if_OrientRotate"); r.eol();
    for (int i = 0; i < 3; i++) { r.get(d.Tg2c[i][0], "Tg2c").get(d.Tg2c[i][1], "Tg2c").get(d.Tg2c[i][2], "Tg2c"); r.eol(); }
    r.get(d.theta_mag, "theta_mag").get(d.phi_mag, "phi_mag"); r.eol();
    r.get(d.px_init, "px").get(d.py_init, "py").get(d.pz_init, "pz"); r.eol();
    r.flag(d.read_Hext_nonunif, "if_read_Hext_nonunif"); r.eol();
    for (int i = 0; i < 3; i++) r.get(d.Hext_stat[i], "Hext_stat"); r.eol();
    for (int i = 0; i < 3; i++) r.get(d.Hext_altr[i], "Hext_altr"); r.eol();
    for (int i = 0; i < 3; i++) r.get(d.H_altr_freq[i], "H_altr_freq"); r.eol();
    r.flag(d.prescribe_H, "if_prescribe_Hext").get(d.n_prescribe_H, "num_prescribe_Hext"); r.eol();
    for (int i = 0; i < 3; i++) r.get(d.Eext_stat[i], "Eext_stat"); r.eol();
    for (int i = 0; i < 3; i++) r.get(d.Eext_altr[i], "Eext_altr"); r.eol();
    for (int i = 0; i < 3; i++) r.get(d.E_altr_freq[i], "E_altr_freq"); r.eol();
    r.flag(d.prescribe_E, "if_prescribe_Eext").get(d.n_prescribe_E, "num_prescribe_Eext"); r.eol();
    r.flag(d.magnetostatics, "if_magnetostatics").flag(d.mag_1D, "if_mag_1Dmodel"); r.eol();
    r.flag(d.demag_factor, "if_demag_factor").get(d.demag_fac[0], "demag_fac_x").get(d.demag_fac[1], "demag_fac_y").get(d.demag_fac[2], "demag_fac_z"); r.eol();
    r.flag(d.elec_1D, "if_elec_1Dmodel").flag(d.elec_1D_comp, "if_elec_1D_compensate"); r.eol();
    r.flag(d.em_dynamic, "if_EMdynamic").flag(d.planeEM, "if_input_planeEM_E"); r.eol();
    for (int i = 0; i < 3; i++) r.get(d.planeEM_E[i], "planeEM_E"); r.eol();
    for (int i = 0; i < 3; i++) r.get(d.planeEM_freq[i], "planeEM_E_freq"); r.eol();
    r.flag(d.em_fromP, "if_EM_fromP").flag(d.em_fromM, "if_EM_fromM"); r.eol();
    r.flag(d.em_back_P, "if_EM_backaction_on_P").flag(d.em_back_M, "if_EM_backaction_on_M"); r.eol();
    r.get(d.free_charge_nzi, "free_charge_nzi").get(d.free_charge_nzf, "free_charge_nzf").get(d.free_charge, "free_charge"); r.eol();
    r.get(d.scale_elec, "scale_elec").get(d.elec_limit, "elec_solver_limit").get(d.elec_tol, "elec_solver_tol"); r.eol();
    r.flag(d.elastodynamics, "if_elastodynamics").flag(d.elasto_back, "if_elasto_backaction_from_pORm").flag(d.elasto_on, "if_elasto_on_pORm"); r.eol();
    r.flag(d.strain_pulse, "if_gaussian_strain_pulse").get(d.strain_type, "input_strain_type").get(d.strain_z, "input_strain_sourcez"); r.eol();
    r.get(d.strain_comp, "input_strain_component").get(d.sigma_gauss, "sigma_gauss").get(d.amp_gauss, "amplitude_gauss").get(d.strain_cycles, "num_strain_cycles"); r.eol();
    r.flag(d.elastostatic, "if_elastostatic").flag(d.elastostatic_1D, "if_elastostatic_1D"); r.eol();
    r.flag(d.read_strain_ext, "if_read_strain_ext").flag(d.elastostatic_film, "if_elastostatic_film"); r.eol();
    r.get(d.strain_ext_nzi, "strain_ext_nzi").get(d.strain_ext_nzf, "strain_ext_nzf").get(d.exx_ext, "exx_ext").get(d.eyy_ext, "eyy_ext").get(d.exy_ext, "exy_ext"); r.eol();
    r.get(d.scale_elasto, "scale_elasto").get(d.elasto_limit, "elasto_solver_limit").get(d.elasto_tol, "elasto_solver_tol"); r.eol();
    r.flag(d.abc_1D, "if_1D_ABC").flag(d.abc_elast_onlytop, "if_1D_ABC_ELAST_onlytop").flag(d.abc_em_onlytop, "if_1D_ABC_EM_onlytop").get(d.liao_w, "weighting_factor_fourth_Liao"); r.eol();
    r.flag(d.pec_xy, "if_PEC_XY").flag(d.pec_z, "if_PEC_Z"); r.eol();
    r.flag(d.flexo, "if_flexo"); r.eol();
    r.flag(d.spin_pumping, "if_spin_pumping"); r.eol();
    r.flag(d.in_m, "if_input_m").flag(d.in_afm, "if_input_AFMm").flag(d.in_Hstat, "if_input_Hstat"); r.eol();
    r.flag(d.in_pq, "if_input_pandq").flag(d.in_Estat, "if_input_Estat"); r.eol();
    r.flag(d.in_em, "if_input_em").flag(d.in_Jp, "if_input_Jp"); r.eol();
    r.flag(d.in_uv, "if_input_uandv").flag(d.in_straint0, "if_input_straint0").flag(d.in_eig0, "if_input_eigenstraint0_crt"); r.eol();
    r.flag(d.in_force, "if_input_elastoforce"); r.eol();
    // output schedule (gf_write_outputs / gf_run_deck write these files)
    {
        auto out = [&](Deck::Out& o, const char* flag, const char* step) -> Reader& { return r.flag(o.on, flag).get(o.step, step); };
        out(d.out_ave, "if_output_ave", "output_step_ave"); r.eol();
        out(d.out_m, "if_output_m", "output_step_m");
        out(d.out_magcell, "if_output_only_magcell", "output_step_magcell"); r.eol();
        out(d.out_AFMm, "if_output_AFMm", "output_step_AFMm"); r.eol();
        out(d.out_p, "if_output_p", "output_step_p"); r.eol();
        out(d.out_em, "if_output_em", "output_step_em");
        out(d.out_em_onecell, "if_output_em_onecell", "output_step_em_onecell").get(d.em_onecell_index, "em_onecell_index"); r.eol();
        struct NO { Deck::Out* o; const char* name; } rest[] = {
            {&d.out_strain, "if_output_strain"}, {&d.out_Hstat, "if_output_Hstat"}, {&d.out_Estat, "if_output_Estat"},
            {&d.out_eig0, "if_output_eigenstraint0_crt"}, {&d.out_q, "if_output_q"}, {&d.out_uv, "if_output_uandv"},
            {&d.out_force, "if_output_elastoforce"}, {&d.out_emYee, "if_output_emYee"}, {&d.out_Jp, "if_output_Jp"},
            {&d.out_Jishe, "if_output_Jishe"}};
        for (const NO& no : rest) { out(*no.o, no.name, "output step"); r.eol(); }
    }
    r.flag(d.jf_input, "if_Jf_input"); r.eol();
    r.get(d.jf_i0, "Jfin_xi").get(d.jf_j0, "Jfin_yi").get(d.jf_k0, "Jfin_zi"); r.eol();
    r.get(d.jf_i1, "Jfin_xf").get(d.jf_j1, "Jfin_yf").get(d.jf_k1, "Jfin_zf"); r.eol();
    r.get(d.jf_type, "Jf_input_type").get(d.jf_comp, "Jf_input_component").get(d.jf_amp, "Jf_input_amp").get(d.jf_freq, "Jf_input_freq").get(d.jf_sigma, "Jf_input_sigma").get(d.jf_cycles, "num_Jf_cycles"); r.eol();
    r.flag(d.prescribed_m, "if_prescribed_m").get(d.precess_angle, "precess_angle").get(d.precess_freq, "precess_frequency"); r.eol();
    if (!r.err.empty()) return r.err;
    r.f.close();

    // Tc2g = transpose(Tg2c) (read.cpp:105-107)
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) d.Tc2g[i][j] = d.Tg2c[j][i];

    std::string e = read_materials(dir, d);
    if (!e.empty()) return e;

    for (unsigned v : d.material_layer_unit)
        if (v > d.num_materials) return "layer material id exceeds num_materials";
    if (d.id_firstlayer < 1 || d.id_lastlayer_unit < d.id_firstlayer || d.id_lastlayer_unit > d.num_layer_unit)
        return "bad layer-unit ids";
    if (d.nx_work > d.nx || d.ny_work > d.ny || d.nx_work < 0 || d.ny_work < 0) return "work region larger than the grid";
    expand_layers(d);
    if (d.idzf > d.nz - 1) return "layers are thicker than nz";

    if (d.read_struct) {
        std::ifstream f(dir + "/struct.in");
        if (f.is_open()) {
            for (long i = 0; i < d.n(); i++) {
                unsigned long x, y, z, id;
                f >> x >> y >> z >> id;
                if (f.fail()) return "malformed struct.in";
                if (x < 1 || y < 1 || z < 1 || (long)x > d.nx || (long)y > d.ny || (long)z > d.nz || id > d.num_materials)
                    return "struct.in entry out of range";
                d.material_cell[(size_t)(((x - 1) * d.ny + (y - 1)) * d.nz + (z - 1))] = (uint8_t)id;
            }
        }
    }

    finish_deck(d);
    if (d.prescribe_E) { e = read_table(dir + "/Eext.in", d.n_prescribe_E, d.tE, d.Ex, d.Ey, d.Ez); if (!e.empty()) return e; }
    if (d.prescribe_H) { e = read_table(dir + "/Hext.in", d.n_prescribe_H, d.tH, d.Hx, d.Hy, d.Hz); if (!e.empty()) return e; }
    return "";
}

std::string deck_from_params(const gf_run_params& r, const gf_material_params* mats, int nmat,
                             const uint32_t* material_cell, Deck& d) {
    if (r.nx < 1 || r.ny < 1 || r.nz < 1) return "grid dimensions must be positive";
    if (!(r.dx > 0. && r.dy > 0. && r.dz > 0.)) return "cell sizes must be positive";
    if (nmat < 1 || nmat > 255) return "n_materials must be 1..255";
    if (!mats || !material_cell) return "null materials or material_cell";
    d = Deck();
    d.nx = r.nx; d.ny = r.ny; d.nz = r.nz;
    d.dx = r.dx; d.dy = r.dy; d.dz = r.dz;
    d.per_x = r.periodicX != 0; d.per_y = r.periodicY != 0; d.per_z = r.periodicZ != 0;
    d.nx_work = r.nx; d.ny_work = r.ny;
    d.steps = r.step; d.dt = r.dt;
    d.num_materials = (unsigned)nmat;
    d.orient_rotate = r.if_OrientRotate != 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) d.Tg2c[i][j] = r.Tg2c[i][j];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) d.Tc2g[i][j] = d.Tg2c[j][i];
    d.theta_mag = r.theta_mag; d.phi_mag = r.phi_mag;
    d.px_init = r.px_init; d.py_init = r.py_init; d.pz_init = r.pz_init;
    for (int a = 0; a < 3; a++) {
        d.Hext_stat[a] = r.Hext_stat[a]; d.Hext_altr[a] = r.Hext_altr[a]; d.H_altr_freq[a] = r.H_altr_freq[a];
        d.Eext_stat[a] = r.Eext_stat[a]; d.Eext_altr[a] = r.Eext_altr[a]; d.E_altr_freq[a] = r.E_altr_freq[a];
        d.demag_fac[a] = r.demag_fac[a];
        d.planeEM_E[a] = r.planeEM_E[a]; d.planeEM_freq[a] = r.planeEM_E_freq[a];
    }
    d.prescribe_H = r.if_prescribe_Hext != 0; d.n_prescribe_H = 0;
    d.prescribe_E = r.if_prescribe_Eext != 0; d.n_prescribe_E = 0;
    d.magnetostatics = r.if_magnetostatics != 0; d.mag_1D = r.if_mag_1Dmodel != 0;
    d.demag_factor = r.if_demag_factor != 0;
    d.elec_1D = r.if_elec_1Dmodel != 0; d.elec_1D_comp = r.if_elec_1D_compensate != 0;
    d.scale_elec = r.scale_elec; d.elec_limit = (unsigned)(r.elec_solver_limit > 0 ? r.elec_solver_limit : 0);
    d.elec_tol = r.elec_solver_tol;
    d.em_dynamic = r.if_EMdynamic != 0; d.planeEM = r.if_input_planeEM_E != 0;
    d.em_fromP = r.if_EM_fromP != 0; d.em_fromM = r.if_EM_fromM != 0;
    d.em_back_P = r.if_EM_backaction_on_P != 0; d.em_back_M = r.if_EM_backaction_on_M != 0;
    d.abc_1D = r.if_1D_ABC != 0; d.abc_elast_onlytop = r.if_1D_ABC_ELAST_onlytop != 0;
    d.abc_em_onlytop = r.if_1D_ABC_EM_onlytop != 0; d.liao_w = r.weighting_factor_fourth_Liao;
    d.pec_xy = r.if_PEC_XY != 0; d.pec_z = r.if_PEC_Z != 0;
    d.jf_input = r.if_Jf_input != 0;
    if (d.jf_input) {
        for (int a = 0; a < 3; a++)
            if (r.Jfin_lo[a] < 0 || r.Jfin_hi[a] < r.Jfin_lo[a]) return "bad J_f box";
        d.jf_i0 = (unsigned long)r.Jfin_lo[0]; d.jf_j0 = (unsigned long)r.Jfin_lo[1]; d.jf_k0 = (unsigned long)r.Jfin_lo[2];
        d.jf_i1 = (unsigned long)r.Jfin_hi[0]; d.jf_j1 = (unsigned long)r.Jfin_hi[1]; d.jf_k1 = (unsigned long)r.Jfin_hi[2];
    }
    d.jf_type = (unsigned)(r.Jf_input_type > 0 ? r.Jf_input_type : 0);
    d.jf_comp = r.Jf_input_component ? r.Jf_input_component : 'x';
    d.jf_amp = r.Jf_input_amp; d.jf_freq = r.Jf_input_freq; d.jf_sigma = r.Jf_input_sigma; d.jf_cycles = r.num_Jf_cycles;
    d.elastodynamics = r.if_elastodynamics != 0; d.elasto_back = r.if_elasto_backaction_from_pORm != 0;
    d.elasto_on = r.if_elasto_on_pORm != 0;
    d.strain_pulse = r.if_gaussian_strain_pulse != 0;
    d.strain_type = (unsigned)(r.input_strain_type > 0 ? r.input_strain_type : 0);
    d.strain_z = (unsigned)(r.input_strain_sourcez > 0 ? r.input_strain_sourcez : 0);
    d.strain_comp = r.input_strain_component ? r.input_strain_component : 'x';
    d.sigma_gauss = r.sigma_gauss; d.amp_gauss = r.amplitude_gauss; d.strain_cycles = r.num_strain_cycles;
    d.elastostatic = r.if_elastostatic != 0; d.flexo = r.if_flexo != 0; d.prescribed_m = r.if_prescribed_m != 0;
    d.spin_pumping = r.if_spin_pumping != 0;
    d.scale_elasto = r.scale_elasto; d.elasto_limit = (unsigned)r.elasto_solver_limit; d.elasto_tol = r.elasto_solver_tol;

    d.mats.assign((size_t)nmat, Material());
    for (int i = 0; i < nmat; i++) {
        const gf_material_params& s = mats[i];
        Material& m = d.mats[i];
        m.c11 = s.c11; m.c12 = s.c12; m.c44 = s.c44; m.density = s.density;
        m.mass_damping = s.elast_mass_damping; m.stiff_damping = s.elast_stiff_damping;
        m.fm = s.if_FM != 0; m.Ms = s.Ms; m.gyro = s.gyro; m.alpha = s.FM_damping;
        m.aniso_type = (unsigned)(s.anisotropy_type > 0 ? s.anisotropy_type : 0);
        m.K1 = s.K1; m.K2 = s.K2; m.Aex = s.Aex; m.iDMI = s.iDMI; m.lam100 = s.lamda100; m.lam111 = s.lamda111;
        m.afm = s.if_AFM != 0;
        m.Ms1 = s.Ms_AFM[0]; m.Ms2 = s.Ms_AFM[1]; m.gyro1 = s.gyro_AFM[0]; m.gyro2 = s.gyro_AFM[1];
        m.alpha1 = s.damping_AFM[0]; m.alpha2 = s.damping_AFM[1]; m.K1_1 = s.K1_AFM[0]; m.K1_2 = s.K1_AFM[1];
        {
            // read.cpp:149-153
            const double norm = std::sqrt(s.uniaxis_AFM[0] * s.uniaxis_AFM[0] + s.uniaxis_AFM[1] * s.uniaxis_AFM[1] +
                                          s.uniaxis_AFM[2] * s.uniaxis_AFM[2]);
            for (int a = 0; a < 3; a++) m.uaxis[a] = s.uniaxis_AFM[a] / norm;
        }
        m.Aex1 = s.Aex_AFM[0]; m.Aex2 = s.Aex_AFM[1]; m.J_AFM = s.J_AFM;
        m.lam100_1 = s.lamda100_AFM[0]; m.lam100_2 = s.lamda100_AFM[1];
        m.lam111_1 = s.lamda111_AFM[0]; m.lam111_2 = s.lamda111_AFM[1];
        m.spin_pump = s.if_spin_pump != 0;
        m.sh_angle = s.spin_hall_angle; m.sh_mixcond = s.spin_mix_cond; m.sh_difflen = s.spin_diffus_length;
        m.fe = s.if_FE != 0; m.fe_mass = s.FE_mass; m.fe_damping = s.FE_damping;
        m.a1 = s.a1; m.a11 = s.a11; m.a12 = s.a12; m.a111 = s.a111; m.a112 = s.a112; m.a123 = s.a123;
        m.a1111 = s.a1111; m.a1112 = s.a1112; m.a1122 = s.a1122; m.a1123 = s.a1123;
        m.G11 = s.G11; m.Q11 = s.Q11; m.Q12 = s.Q12; m.Q44 = s.Q44; m.f11 = s.f11; m.f12 = s.f12; m.f44 = s.f44;
        m.pec = s.if_PEC != 0; m.er = s.r_permittivity; m.cond = s.conductivity;
        for (int k = 0; k < 3; k++) { m.comp[k] = s.comp_n[k]; m.wp[k] = s.omega_plasma_n[k]; m.tau[k] = s.tao_e_n[k]; }
        derive_material(m, d.Tc2g);
    }
    d.material_cell.assign((size_t)d.n(), 0);
    for (long c = 0; c < d.n(); c++) {
        if (material_cell[c] > (uint32_t)nmat) return "material_cell id exceeds n_materials";
        d.material_cell[(size_t)c] = (uint8_t)material_cell[c];
    }
    finish_deck(d);
    return "";
}


std::string read_restart(const std::string& path, long nx, long ny, long nz, int ncomp, std::vector<double>* comps) {
    std::ifstream f(path);
    if (!f.is_open()) return "";
    const long n = nx * ny * nz;
    for (long i = 0; i < n; i++) {
        long x, y, z;
        f >> x >> y >> z;
        double v[9];
        for (int c = 0; c < ncomp; c++) f >> v[c];
        if (f.fail()) return "malformed restart file " + path;
        if (x < 1 || y < 1 || z < 1 || x > nx || y > ny || z > nz) return "index out of range in " + path;
        long id = ((x - 1) * ny + (y - 1)) * nz + (z - 1);
        for (int c = 0; c < ncomp; c++) comps[c][(size_t)id] = v[c];
    }
    return "";
}

}  // namespace gf
