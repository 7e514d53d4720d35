// qp_driver: QUILL's driver (src/main.cpp) for one GPU region, on top of the
// libquill_b200 C ABI.
//
//   python3 <quill>/parse.py <conf> | qp_driver
//
// Reads the record stream QUILL's parse.py writes (name, value, units, "$"
// per record, a lone "$" at the end; var::read, low-level.cpp:376-451), with
// QUILL's parameter names, units and defaults for the supported subset
// (below), builds the initial laser field (f_init_cos with the default
// cos envelope, init.cpp:6-210) and the plasma films (film /
// fill_cell_by_particles, init.cpp:402-646), runs the time loop of
// main.cpp:2319-2432 through qp_step and writes QUILL's output files in its
// formats so that python/resread.py reads them (the list is below).
//
// Supported parameters: dx dy dz dt (either may be left out: automatic dx / dt
// as main.cpp:2600-2615) lambda (cm, um, lambda_p) ne xlength ylength zlength
// t_end output_period a0 a0y a0z P I W polarization xsigma ysigma zsigma x0
// y0 z0 x0fout phase
// f_envelope (cos | sscos | pearl | tophat | uniformB | focused |
// focussedSSC) shenergy shphase phi_rotate r0 theta
// xtarget ytarget ztarget lp_reflection f_reflection beam beam_particles Nb
// epsb xb rb x0b y0b phib
// b_sign phi external_bz solver pusher qed film x0film filmwidth gradwidth
// y0film y1film z0film z1film nfilm mcr Tfilm vxfilm xnpic_film ynpic_film
// znpic_film xnpic ynpic znpic ions data_folder output_mode
// e_components_for_output b_components_for_output particles_for_output enthp
// pmerging crpc mwindow (off | on | auto) mwtolerance mwspeed mwseed
// mwseed_ions mw_mcr t_add_mw ne_profile_x_coords ne_profile_x_values
// ne_profile_r_coords ne_profile_r_values nfilm_y0 nfilm_y1 gradwidth_y
// nelflow vlflow mcrlflow Tlflow nerflow vrflow mcrrflow Trflow catching
// dump_photons n_tracks particles_to_track tr_init tr_start xtr1 ytr1 ztr1
// xtr2 ytr2 ztr2 deps deps_p deps_ph deps_i neps neps_p neps_ph neps_i
// enthp_p enthp_ph enthp_i j_components_for_output balancing_particle_weight
// and three additions: precision (fp64 | mixed), seed, and current_order
// (atomic | reference: J summed in the reference's order, FP64, QED off).
//
// Output files: log, N, energy, ex..bz, jx..jz (scaled by dx/dt), w, inv,
// rho, rho_p, rho_ph, irho_<mcr>_, spectrum, spectrum_p, spectrum_ph,
// spectrum_<mcr>_, phasespace, phasespace_p, phasespace_ph,
// phasespace_<mcr>_, weights, mwcoordinate, energy_deleted, deleted*,
// spectrum_deleted_ph, track files, each as the reference writes it.
//
//   qp_driver --initial-fields <file>
//
// stops after the initial fields (laser and beam fields, before any GPU
// work) and writes them to <file>: Ex Ey Ez Bx By Bz, each nx*ny*nz doubles
// with k fastest.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "quill_b200.h"

namespace {

const double PI = 3.141592653589793;
const double PROTON_MASS = 1836.1526721;  // include/physical_constants.h

// ---------------------------------------------------------------- input ----
struct Var {
    std::string name;
    double value = 0;
    std::string units;
    std::vector<double> arr;  // "[a;b;c]" values (input_array)
};

// One record: name, value (or '#'), units or text (or '#'), '$'.
std::vector<Var> read_stream(std::istream& in) {
    std::vector<Var> vars;
    std::string name;
    while (in >> name) {
        if (name == "$") break;
        std::string val, units, end;
        in >> val >> units >> end;
        if (end != "$") throw std::runtime_error("malformed record for " + name);
        Var v;
        v.name = name;
        if (!val.empty() && val[0] == '[') {
            // an array: numbers separated by ';' up to ']' (atof, low-level.cpp:387-411)
            std::string cur;
            for (size_t i = 1; i < val.size() && val[i] != ']'; i++) {
                if (val[i] == ';') { v.arr.push_back(std::atof(cur.c_str())); cur.clear(); }
                else cur += val[i];
            }
            if (!cur.empty()) v.arr.push_back(std::atof(cur.c_str()));
        } else {
            // the reference reads a single value with stof (low-level.cpp:414): float precision
            v.value = (val == "#" || val.empty()) ? 0.0 : (double)std::stof(val);
        }
        v.units = units == "#" ? "" : units;
        vars.push_back(v);
    }
    return vars;
}

// find (low-level.cpp:453-471): first record with this name at or after
// position `from`, else an empty record.
const Var& find(const std::vector<Var>& v, const std::string& n, size_t from = 0, size_t* at = nullptr) {
    static const Var empty;
    for (size_t i = from; i < v.size(); i++)
        if (v[i].name == n) {
            if (at) *at = i;
            return v[i];
        }
    if (at) *at = v.size();
    return empty;
}

// lengths: um / fs / lambda -> c/omega (main.cpp:2616-2650 pattern)
double length(const Var& v, double lambda_cm) {
    double x = v.value;
    if (v.units == "um") x = x * 1e-4 / lambda_cm;
    else if (v.units == "fs") x = x * 1e-15 * 2.99792458e10 / lambda_cm;
    return x * 2 * PI;
}

// ------------------------------------------------------------ parameters ---
struct Film {
    double x0 = 0, width = 0, grad = 0, y0 = 0, y1 = 0, z0 = 0, z1 = 0, ne = 0, mcr = 1, T = 0, vx = 0;
    double ne_y0 = 0, ne_y1 = 0, grad_y = 0;  // cm^-3 at y0film / y1film, 1/k
    int xn = 0, yn = 0, zn = 0;
};

// a neutral flow entering through a face (main.cpp:1837-1880); n in n_cr
struct Flow {
    double n = 0, v = 0, mcr = 0, T = 0;
};

struct Config {
    double dx, dy, dz, dt, lambda, ne = 0, xlength, ylength, zlength;
    std::vector<double> t_end, output_period;
    double a0y = 0, a0z = 0, xsigma = 0, ysigma = 0, zsigma = 0, x0 = 0, y00 = 0, z00 = 0, phase = 0, phi = 0;
    int sscos = 0;                 // f_envelope: cos 0, sscos 1, pearl 2, tophat 3 (main.cpp:2811-2825)
    bool uniform_b = false;        // f_envelope = uniformB (init.cpp:387-400)
    bool focused = false;          // f_envelope = focused / focussedSSC (main.cpp:2906-2925)
    double sigma0 = 0;             // focused: the waist, (ysigma + zsigma) / 2
    double shenergy = 0, shphase = 0;  // focused: second-harmonic energy share and phase (main.cpp:2926-2931)
    double phi_rotate = 0, xtarget = 0, ytarget = 0, ztarget = 0;  // main.cpp:2835-2899
    std::string lp_reflection = "off", f_reflection = "off";        // main.cpp:3402-3407
    bool beam = false;             // main.cpp:2988-3053
    std::string beam_particles = "e";
    double Nb = 0, epsb = 0, xb = 0, rb = 0, x0b = 0, y0b = 0, phib = 0;
    bool b_sign = true;
    double external_bz = 0;
    int solver = QP_SOLVER_NDFX, pusher = QP_PUSHER_VAY;
    bool qed = true;
    std::vector<Film> films;
    std::string ions = "off";
    int xnpic = 1, ynpic = 1, znpic = 1;
    std::string data_folder = "results";
    bool binary = false;
    std::string e_out = "y", b_out = "z", particles_for_output = "e";
    int enthp = 1;
    int precision = QP_PREC_FP64;
    uint64_t seed = 0;
    std::string polarization = "linear";
    bool mwindow = false;          // main.cpp:2932-2938
    bool mw_auto = false;          // mwindow = auto (main.cpp:1961-1975)
    double mwtolerance = 1e-6;     // main.cpp:2939-2943
    bool mwseed_ions = false;      // main.cpp:2951-2954
    double mw_mcr = 1;             // main.cpp:2955-2958
    std::vector<double> prof_x, prof_xv, prof_r, prof_rv;  // ne_profile_* (main.cpp:3496-3523), coords in 1/k
    Flow lflow, rflow;             // nelflow ... Trflow (main.cpp:3232-3249)
    double mwspeed = 1;            // main.cpp:2944-2947
    bool mwseed = true;            // main.cpp:2948-2950
    double t_add_mw = 0;           // main.cpp:2665-2679, 1/omega (0: last output time)
    bool catching = false;         // main.cpp:3531-3534
    bool dump_photons = false;     // emitted photons deleted as they are born
    int n_tracks = 0;              // main.cpp:3408-3413
    std::string particles_to_track = "epgi";
    bool tr_volume = false;        // tr_init = volume: n_tracks random cells in the box (main.cpp:1612-1690)
    double tr_start = 0, xtr1 = 0, ytr1 = 0, ztr1 = 0, xtr2 = 0, ytr2 = 0, ztr2 = 0;  // main.cpp:3419-3480
    double deps = 0, deps_p = 0, deps_ph = 0, deps_i = 0;  // MeV (MeV per nucleon for ions), spectrum bins
                                   // (main.cpp:3337-3362)
    int neps = 0, neps_p = 0, neps_ph = 0, neps_i = 0;      // spectrum bins (main.cpp:3363-3373)
    bool write_p = false, write_ph = false;  // particles_for_output ep / eph / epph (main.cpp:3390-3395)
    bool write_j[3] = {false, false, false};  // j_components_for_output (main.cpp:2961-2978)
    double x0fout = 0;             // yz plane of the field/density files at xlength - x0fout (main.cpp:2718-2731)
    double balancing_particle_weight = 3.0;  // layer weights (main.cpp:3599)
    bool ordered_current = false;  // addition: current_order = reference (J summed in the reference's order)
    int enthp_p = 0, enthp_ph = 0, enthp_i = 0;  // main.cpp:3374-3385
    std::string pmerging = "off";  // off | ti | nl (main.cpp:3397-3399)
    double crpc = 0;               // critical macro-particles per cell (main.cpp:3400-3401)
};

Config parse(const std::vector<Var>& v) {
    Config c;
    c.dx = find(v, "dx").value * 2 * PI;
    c.dy = find(v, "dy").value * 2 * PI;
    c.dz = find(v, "dz").value * 2 * PI;
    c.dt = find(v, "dt").value * 2 * PI;
    Var lam = find(v, "lambda");
    c.lambda = lam.units == "um" ? lam.value * 1e-4 : lam.value;  // cm
    Var ne = find(v, "ne");
    c.ne = ne.units == "ncr" ? ne.value * 1.11485e+13 / c.lambda / c.lambda : ne.value;
    // lambda in units of the plasma wavelength (main.cpp:2593-2599)
    if (lam.units == "lambda_p") c.lambda = lam.value * std::sqrt(1.11485e13 / c.ne);
    if (!(c.lambda > 0)) throw std::runtime_error("lambda must be given");
    // automatic dt and dx (main.cpp:2600-2615): dt half the critical step of
    // the plasma of density ne, dx the least dispersive stable step for dt
    if (c.dt == 0 || c.dx == 0) {
        if (!(c.ne > 0)) throw std::runtime_error("automatic dt / dx need ne");
        const double k0 = std::sqrt(1.11485e+13 / c.lambda / c.lambda / c.ne);
        if (c.dt == 0) {
            c.dt = 0.5 * k0 * std::sqrt(4.04);
            c.dx = 0;
        }
        if (c.dx == 0) {
            c.dx = (1 + 1e-4) * c.dt / (1 - 1 / (k0 * k0) * c.dt * c.dt / 4.04);
            if (c.dx < 0) throw std::runtime_error("Cannot calculate stable dx, reduce dt");
        }
    }
    if (!(c.dx > 0 && c.dy > 0 && c.dz > 0 && c.dt > 0)) throw std::runtime_error("dy and dz must be given");
    auto len_lambda = [&](const char* n) {
        Var x = find(v, n);
        if (x.units == "um") return x.value * 1e-4 / c.lambda * 2 * PI;
        if (x.units == "fs") return x.value * 1e-15 * 2.99792458e10 / c.lambda * 2 * PI;
        return x.value * 2 * PI;
    };
    c.xlength = len_lambda("xlength");
    c.ylength = len_lambda("ylength");
    c.zlength = len_lambda("zlength");
    // t_end / output_period pairs (main.cpp:2652-2662)
    size_t pos = 0;
    while (true) {
        size_t at;
        const Var& te = find(v, "t_end", pos, &at);
        if (at >= v.size() || te.value == 0) break;
        double t = te.value * 2 * PI;
        if (te.units == "um") t = te.value * 1e-4 / c.lambda * 2 * PI;
        if (te.units == "fs") t = te.value * 1e-15 * 2.99792458e10 / c.lambda * 2 * PI;
        size_t at2;
        const Var& op = find(v, "output_period", at + 1, &at2);
        double per = op.units == "t_end" ? op.value * t : op.value * 2 * PI;
        if (!(per > 0)) per = t;
        c.t_end.push_back(t);
        c.output_period.push_back(per);
        pos = at + 1;
    }
    if (c.t_end.empty()) throw std::runtime_error("t_end must be given");
    // laser amplitude and polarisation (main.cpp:2727-2805)
    c.xsigma = length(find(v, "xsigma"), c.lambda);
    c.ysigma = length(find(v, "ysigma"), c.lambda);
    c.zsigma = length(find(v, "zsigma"), c.lambda);
    c.x0 = length(find(v, "x0"), c.lambda);
    c.y00 = length(find(v, "y0"), c.lambda);
    c.z00 = length(find(v, "z0"), c.lambda);
    c.x0fout = length(find(v, "x0fout"), c.lambda);
    if (c.x0fout == 0) c.x0fout = c.xlength / 2;
    // the amplitude from the power, the intensity or the energy
    // (main.cpp:2735-2771); a0 given explicitly wins
    {
        const Var& P = find(v, "P");
        double pv = P.value;
        if (P.units == "PW") pv *= 1e22;
        if (P.units == "TW") pv *= 1e19;
        if (pv != 0) c.a0y = 5.27281e+17 * std::sqrt(2 * pv / (PI * 2.42161e+52 * c.ysigma * c.zsigma));
        const Var& I = find(v, "I");
        double iv = I.value;
        if (I.units == "W/cm^2") iv *= 1e7;
        if (iv != 0) c.a0y = 5.27281e+17 * c.lambda * std::sqrt(iv / (PI * 2.42161e+52));
        const Var& W = find(v, "W");
        double wv = W.value;
        if (W.units == "J") wv *= 1e7;
        if (wv != 0) {
            // 3.691e4 = (mc^2)^2/(8 pi^2 e^2)
            c.a0y = std::sqrt(wv / (3.691e4 * c.lambda * PI * std::sqrt(PI / 2) * c.xsigma * c.ysigma * c.zsigma / 4));
            if (find(v, "polarization").units == "circular") {
                c.a0y = c.a0y / std::sqrt(2);
                c.a0z = c.a0y;
            }
        }
    }
    if (find(v, "a0").value != 0) c.a0y = find(v, "a0").value;
    const Var& pol = find(v, "polarization");
    if (pol.units == "circular") { c.a0z = c.a0y; c.polarization = "circular"; }
    if (pol.units == "elliptic") { c.a0z = pol.value * c.a0y; c.polarization = "elliptic"; }
    if (find(v, "a0y").value != 0) {
        c.a0y = find(v, "a0y").value;
        c.a0z = find(v, "a0z").value;
    } else if (find(v, "a0z").value != 0) {
        c.a0z = find(v, "a0z").value;
        c.a0y = 0;
    }
    const Var& ph = find(v, "phase");
    c.phase = ph.units == "pi" ? ph.value * PI : ph.value;
    c.b_sign = find(v, "b_sign").value != -1;
    const Var& phi = find(v, "phi");
    c.phi = phi.units == "pi" ? phi.value * PI : phi.value;
    const std::string env = find(v, "f_envelope").units;
    if (env.empty() || env == "cos") c.sscos = 0;
    else if (env == "sscos") c.sscos = 1;
    else if (env == "pearl") c.sscos = 2;
    else if (env == "tophat") c.sscos = 3;
    else if (env == "uniformB") c.uniform_b = true;
    else if (env == "focused") c.focused = true;
    else if (env == "focussedSSC") { c.focused = true; c.sscos = 1; }
    else throw std::runtime_error("f_envelope " + env + " is not part of this build (cos, sscos, pearl, tophat, uniformB, focused, focussedSSC)");
    const Var& phr = find(v, "phi_rotate");
    c.phi_rotate = phr.units == "pi" ? phr.value * PI : phr.value;
    // the pulse position as (r0, theta) (main.cpp:2850-2867)
    const Var& r0v = find(v, "r0");
    if (r0v.units != "off" && r0v.value != 0) {
        const double r0 = length(r0v, c.lambda);
        const Var& th = find(v, "theta");
        const double theta = th.units == "deg" ? th.value * PI / 180 : th.value;
        c.x0 = -r0 * std::cos(theta) + 0.00001;
        c.y00 = -r0 * std::sin(theta);
    }
    auto target = [&](const char* n) {
        const Var& x = find(v, n);
        if (x.units == "off" || x.value == 0) return 0.0;
        return x.units == "um" ? x.value * 1e-4 / c.lambda * 2 * PI : x.value * 2 * PI;
    };
    c.xtarget = target("xtarget");
    c.ytarget = target("ytarget");
    c.ztarget = target("ztarget");
    if (c.focused) {
        // the waist from the transverse sizes; the amplitude is given at the
        // focus and scaled to the pulse's starting distance from it
        const double x00 = std::sqrt(c.x0 * c.x0 + c.y00 * c.y00 + c.z00 * c.z00);
        c.sigma0 = 0.5 * (c.ysigma + c.zsigma);
        const double sigma = std::sqrt(c.sigma0 * c.sigma0 + 4 * x00 * x00 / (c.sigma0 * c.sigma0));
        c.a0y = c.a0y * c.sigma0 / sigma;
        c.a0z = c.a0z * c.sigma0 / sigma;
    }
    c.shenergy = find(v, "shenergy").value;
    const Var& shp = find(v, "shphase");
    c.shphase = shp.units == "pi" ? shp.value * PI : shp.value;
    c.lp_reflection = find(v, "lp_reflection").units;
    if (c.lp_reflection.empty()) c.lp_reflection = "off";
    c.f_reflection = find(v, "f_reflection").units;
    if (c.f_reflection.empty()) c.f_reflection = "off";
    // particle beam (main.cpp:2988-3053, init_beam main.cpp:1230-1239)
    c.beam = find(v, "beam").units == "on";
    c.beam_particles = find(v, "beam_particles").units;
    if (c.beam_particles.empty()) c.beam_particles = "e";
    c.Nb = find(v, "Nb").value;
    const Var& eb = find(v, "epsb");
    c.epsb = eb.units == "mc^2" ? eb.value * 0.511 : eb.value;  // MeV
    c.xb = length(find(v, "xb"), c.lambda);
    c.rb = length(find(v, "rb"), c.lambda);
    c.x0b = length(find(v, "x0b"), c.lambda);
    c.y0b = length(find(v, "y0b"), c.lambda);
    const Var& pb = find(v, "phib");
    c.phib = pb.units == "deg" ? pb.value * PI / 180 : pb.value;
    c.external_bz = find(v, "external_bz").value;
    // solver / pusher / qed (main.cpp:3542-3584); defaults NDFX, Vay, QED on
    const std::string sv = find(v, "solver").units, pu = find(v, "pusher").units;
    if (sv == "fdtd") c.solver = QP_SOLVER_FDTD;
    else if (sv == "five_point") c.solver = QP_SOLVER_FIVE_POINT;
    else if (sv.empty() || sv == "ndfx") c.solver = QP_SOLVER_NDFX;
    else throw std::runtime_error("Solver unknown: " + sv);
    if (pu == "boris") c.pusher = QP_PUSHER_BORIS;
    else if (pu.empty() || pu == "vay") c.pusher = QP_PUSHER_VAY;
    else throw std::runtime_error("Pusher unknown: " + pu);
    const std::string q = find(v, "qed").units;
    c.qed = !(q == "off");
    const std::string mw = find(v, "mwindow").units;
    if (mw != "off" && mw != "on" && mw != "auto" && !mw.empty())
        throw std::runtime_error("mwindow must be off, on or auto");
    c.mwtolerance = find(v, "mwtolerance").value;
    if (c.mwtolerance == 0.0) c.mwtolerance = 1e-6;
    c.mw_mcr = find(v, "mw_mcr").value;
    if (c.mw_mcr == 0) c.mw_mcr = 1;
    c.mwseed_ions = find(v, "mwseed_ions").units == "on";
    if (mw.empty() || mw == "on" || mw == "auto") {  // the reference's default is on
        c.mwindow = true;
        c.mw_auto = mw == "auto";
        c.mwspeed = find(v, "mwspeed").value;
        if (c.mwspeed == 0 && !c.mw_auto) c.mwspeed = 1;
        c.mwseed = find(v, "mwseed").units != "off";
        const Var& ta = find(v, "t_add_mw");
        double tv = ta.value;
        if (ta.units == "um") tv = tv * 1e-4 / c.lambda;
        else if (ta.units == "mm") tv = tv / (10 * c.lambda);
        else if (ta.units == "cm") tv = tv / c.lambda;
        c.t_add_mw = tv * 2 * PI;
    }
    // density profiles of the window's new plasma (main.cpp:3496-3523):
    // coordinates in lambda unless given in um
    auto coords = [&](const char* n) {
        const Var& a = find(v, n);
        std::vector<double> out = a.arr;
        for (double& x : out) x = a.units == "um" ? x * 1e-4 / c.lambda * 2 * PI : x * 2 * PI;
        return out;
    };
    c.prof_x = coords("ne_profile_x_coords");
    c.prof_xv = find(v, "ne_profile_x_values").arr;
    c.prof_r = coords("ne_profile_r_coords");
    c.prof_rv = find(v, "ne_profile_r_values").arr;
    if (c.prof_x.size() != c.prof_xv.size() || c.prof_r.size() != c.prof_rv.size())
        throw std::runtime_error("density profile coordinates and values differ in length");
    if (!std::is_sorted(c.prof_x.begin(), c.prof_x.end()) || !std::is_sorted(c.prof_r.begin(), c.prof_r.end()))
        throw std::runtime_error("density profile coordinates are not sorted");
    // neutral flows (main.cpp:3232-3249); they switch the moving window off
    const double ncr = 1.11485e+13 / c.lambda / c.lambda;
    c.lflow = {find(v, "nelflow").value * c.ne / ncr, find(v, "vlflow").value, find(v, "mcrlflow").value,
               find(v, "Tlflow").value};
    c.rflow = {find(v, "nerflow").value * c.ne / ncr, find(v, "vrflow").value, find(v, "mcrrflow").value,
               find(v, "Trflow").value};
    if (c.lflow.n != 0 || c.rflow.n != 0) c.mwindow = c.mw_auto = false;
    // films (main.cpp:3055-3229)
    c.xnpic = (int)find(v, "xnpic").value; if (c.xnpic <= 0) c.xnpic = 1;
    c.ynpic = (int)find(v, "ynpic").value; if (c.ynpic <= 0) c.ynpic = 1;
    c.znpic = (int)find(v, "znpic").value; if (c.znpic <= 0) c.znpic = 1;
    c.ions = find(v, "ions").units;
    for (size_t i = 0; i < v.size(); i++) {
        if (v[i].name != "film" || v[i].units != "on") continue;
        Film f;
        size_t s = i + 1;
        auto fl = [&](const char* n) { return length(find(v, n, s), c.lambda); };
        f.x0 = fl("x0film");
        f.width = fl("filmwidth");
        f.grad = fl("gradwidth");
        f.y0 = fl("y0film");
        f.y1 = find(v, "y1film", s).value == 0 ? c.ylength : fl("y1film");
        f.z0 = fl("z0film");
        f.z1 = find(v, "z1film", s).value == 0 ? c.zlength : fl("z1film");
        auto dens = [&](const char* nm) {
            const Var& n = find(v, nm, s);
            return n.units == "ncr" ? n.value * 1.11485e+13 / c.lambda / c.lambda : (n.units == "ne" ? n.value * c.ne : n.value);
        };
        f.ne = dens("nfilm");
        f.ne_y0 = dens("nfilm_y0");
        f.ne_y1 = dens("nfilm_y1");
        if (f.ne != 0) f.ne_y0 = f.ne_y1 = f.ne;  // init_films, main.cpp:1253-1257
        f.grad_y = fl("gradwidth_y");
        f.mcr = find(v, "mcr", s).value == 0 ? 1 : find(v, "mcr", s).value;
        f.T = find(v, "Tfilm", s).value;
        f.vx = find(v, "vxfilm", s).value;
        f.xn = (int)find(v, "xnpic_film", s).value;
        f.yn = (int)find(v, "ynpic_film", s).value;
        f.zn = (int)find(v, "znpic_film", s).value;
        if (f.xn == 0 || f.yn == 0 || f.zn == 0) { f.xn = c.xnpic; f.yn = c.ynpic; f.zn = c.znpic; }
        c.films.push_back(f);
    }
    if (!find(v, "data_folder").units.empty()) c.data_folder = find(v, "data_folder").units;
    c.binary = find(v, "output_mode").units == "binary";
    // field components written (main.cpp:2959-2978); the reference's default is none
    c.e_out = find(v, "e_components_for_output").units;
    c.b_out = find(v, "b_components_for_output").units;
    if (c.e_out.empty()) c.e_out = "none";
    if (c.b_out.empty()) c.b_out = "none";
    {
        const std::string jc = find(v, "j_components_for_output").units;
        for (int a = 0; a < 3; a++) c.write_j[a] = jc.find("xyz"[a]) != std::string::npos;
    }
    if (!find(v, "particles_for_output").units.empty()) c.particles_for_output = find(v, "particles_for_output").units;
    c.write_p = c.particles_for_output == "ep" || c.particles_for_output == "epph";
    c.write_ph = c.particles_for_output == "eph" || c.particles_for_output == "epph";
    if (find(v, "balancing_particle_weight").value != 0 || !find(v, "balancing_particle_weight").units.empty())
        c.balancing_particle_weight = find(v, "balancing_particle_weight").value;
    c.ordered_current = find(v, "current_order").units == "reference";
    c.enthp = (int)find(v, "enthp").value; if (c.enthp <= 0) c.enthp = 1;
    c.enthp_p = (int)find(v, "enthp_p").value; if (c.enthp_p == 0) c.enthp_p = c.enthp;
    c.enthp_ph = (int)find(v, "enthp_ph").value; if (c.enthp_ph == 0) c.enthp_ph = c.enthp;
    c.enthp_i = (int)find(v, "enthp_i").value; if (c.enthp_i == 0) c.enthp_i = c.enthp;
    c.catching = find(v, "catching").units == "on";
    c.n_tracks = (int)find(v, "n_tracks").value;
    c.particles_to_track = find(v, "particles_to_track").units;
    if (c.particles_to_track.empty()) c.particles_to_track = "epgi";
    if (c.particles_to_track == "none") c.particles_to_track = "";
    c.tr_volume = find(v, "tr_init").units == "volume";  // main.cpp:3414-3418
    {
        const Var& ts = find(v, "tr_start");
        double tv = ts.value;
        if (ts.units == "um") tv = tv * 1e-4 / c.lambda;
        else if (ts.units == "mm") tv = tv / 10 / c.lambda;
        else if (ts.units == "cm") tv = tv / c.lambda;
        c.tr_start = tv * 2 * PI;
    }
    c.xtr1 = length(find(v, "xtr1"), c.lambda); c.ytr1 = length(find(v, "ytr1"), c.lambda); c.ztr1 = length(find(v, "ztr1"), c.lambda);
    c.xtr2 = length(find(v, "xtr2"), c.lambda); c.ytr2 = length(find(v, "ytr2"), c.lambda); c.ztr2 = length(find(v, "ztr2"), c.lambda);
    c.dump_photons = find(v, "dump_photons").units == "on" && c.qed;  // main.cpp:3545-3549
    // spectra (main.cpp:3337-3373): bin widths in MeV (MeV per nucleon for
    // ions), bin counts; each falls back to deps / neps
    auto mev = [&](const char* n) { const Var& w = find(v, n); return w.units == "mc^2" ? w.value * 0.511 : w.value; };
    c.deps = mev("deps");
    c.deps_p = mev("deps_p");
    if (c.deps_p == 0) c.deps_p = c.deps;
    c.deps_ph = mev("deps_ph");
    if (c.deps_ph == 0) c.deps_ph = c.deps;
    c.deps_i = find(v, "deps_i").value;
    if (c.deps_i == 0) c.deps_i = c.deps;
    c.neps = (int)find(v, "neps").value;
    c.neps_p = (int)find(v, "neps_p").value;
    if (c.neps_p == 0) c.neps_p = c.neps;
    c.neps_ph = (int)find(v, "neps_ph").value;
    if (c.neps_ph == 0) c.neps_ph = c.neps;
    c.neps_i = (int)find(v, "neps_i").value;
    if (c.neps_i == 0) c.neps_i = c.neps;
    const std::string pr = find(v, "precision").units;
    if (pr == "mixed") c.precision = QP_PREC_MIXED;
    c.seed = (uint64_t)find(v, "seed").value;
    c.pmerging = find(v, "pmerging").units;
    if (c.pmerging.empty()) c.pmerging = "off";
    if (c.pmerging != "off" && c.pmerging != "ti" && c.pmerging != "nl")
        throw std::runtime_error("pmerging must be off, ti or nl");
    c.crpc = find(v, "crpc").value;
    return c;
}

// --------------------------------------------------------- initial state ---
struct Grid3 {
    int nx, ny, nz;
    long nc() const { return (long)nx * ny * nz; }
    long at(int i, int j, int k) const { return ((long)i * ny + j) * nz + k; }
};

// f_init_cos with the cos envelope (sscos = 0) and append = true
// (init.cpp:6-210): the pulse frame r0 points from (x1, y0, z0) towards the
// box centre; E and B of the envelope-modulated wave are rotated into the box.
void laser_cos(const Config& c, const Grid3& g, std::vector<double>* F, double a0y, double a0z, double xc,
               double x1, double y0, double z0, double phi) {
    double xs = 0, ys = 0, zs = 0;
    if (c.sscos == 0) {
        xs = c.xsigma * 2 * std::sqrt(2 * PI) / 3;
        ys = c.ysigma * 2 * std::sqrt(2 * PI) / 3;
        zs = c.zsigma * 2 * std::sqrt(2 * PI) / 3;
    } else if (c.sscos == 1) {
        xs = 0.822 * c.xsigma; ys = 0.822 * c.ysigma; zs = 0.822 * c.zsigma;
    } else if (c.sscos == 2) {
        xs = c.xsigma * 2 * std::sqrt(2 * PI) / 3; ys = 1e2 * c.ysigma; zs = 1e2 * c.ysigma;
    } else {
        xs = c.xsigma * 2 * std::sqrt(2 * PI) / 3; ys = 0.822 * c.ysigma; zs = 0.822 * c.zsigma;
    }
    const double y12 = 0.5 * g.ny * c.dy, z12 = 0.5 * g.nz * c.dz;
    double r0x = std::sqrt(x1 * x1 + y0 * y0 + z0 * z0);
    double r0y = -y0 / r0x, r0z = -z0 / r0x;
    r0x = -x1 / r0x;
    double y0x, y0y, y0z = std::sqrt(r0x * r0x + r0y * r0y);
    if (y0z != 0) { y0x = -r0y / y0z; y0y = r0x / y0z; y0z = 0; }
    else { y0x = 0; y0y = 1; y0z = 0; }
    double z0x = r0y * y0z - r0z * y0y, z0y = r0z * y0x - r0x * y0z, z0z = r0x * y0y - r0y * y0x;
    if (phi != 0) {
        const double cs = std::cos(phi), sn = std::sin(phi);
        const double yx = y0x, yy = y0y, yz = y0z, zx = z0x, zy = z0y, zz = z0z;
        y0x = yx * cs + zx * sn; y0y = yy * cs + zy * sn; y0z = yz * cs + zz * sn;
        z0x = zx * cs - yx * sn; z0y = zy * cs - yy * sn; z0z = zz * cs - yz * sn;
    }
    for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
            for (int k = 0; k < g.nz; k++) {
                const double X = i * c.dx - xc - c.xtarget, Y = j * c.dy - y12 - y0 - c.ytarget,
                             Z = k * c.dz - z12 - z0 - c.ztarget;
                const double x = r0x * X + r0y * Y + r0z * Z;
                const double y = y0x * X + y0y * Y + y0z * Z;
                const double z = z0x * X + z0y * Y + z0z * Z;
                if (!(x < xs && x > -xs && y < ys && y > -ys && z < zs && z > -zs)) continue;
                const double xi = x + c.phase;
                double ex = 0, ey = 0, ez = 0, bx = 0, by = 0, bz = 0;
                if (c.sscos == 0) {
                    const double cosx = std::cos(PI * x / 2 / xs), cosy = std::cos(PI * y / 2 / ys), cosz = std::cos(PI * z / 2 / zs);
                    const double sinx = std::sin(PI * x / 2 / xs), siny = std::sin(PI * y / 2 / ys), sinz = std::sin(PI * z / 2 / zs);
                    const double tr = cosy * cosy * cosz * cosz;
                    ey = a0y * tr * (std::cos(xi) * cosx * cosx - PI / xs * std::sin(xi) * cosx * sinx);
                    ez = a0z * tr * (std::sin(xi) * cosx * cosx + PI / xs * std::cos(xi) * cosx * sinx);
                    bz = ey; by = -ez;
                    ex = a0y * std::sin(xi) * cosx * cosx * cosz * cosz * PI / ys * cosy * siny -
                         a0z * std::cos(xi) * cosx * cosx * cosy * cosy * PI / zs * cosz * sinz;
                    bx = a0z * std::cos(xi) * cosx * cosx * PI / ys * cosz * cosz * cosy * siny +
                         a0y * std::sin(xi) * cosx * cosx * cosy * cosy * PI / zs * cosz * sinz;
                } else if (c.sscos == 1) {  // super-cosine envelope (init.cpp:122-134)
                    const double x4 = xs * xs * xs * xs, y4 = ys * ys * ys * ys, z4 = zs * zs * zs * zs;
                    const double cosx = std::cos(PI * x * x * x * x / 2 / x4), cosy = std::cos(PI * y * y * y * y / 2 / y4),
                                 cosz = std::cos(PI * z * z * z * z / 2 / z4);
                    const double sinx = std::sin(PI * x * x * x * x / 2 / x4), siny = std::sin(PI * y * y * y * y / 2 / y4),
                                 sinz = std::sin(PI * z * z * z * z / 2 / z4);
                    const double tr = cosy * cosy * cosz * cosz;
                    ey = a0y * tr * (std::cos(xi) * cosx * cosx - 4 * PI * x * x * x / x4 * std::sin(xi) * cosx * sinx);
                    ez = a0z * tr * (std::sin(xi) * cosx * cosx + 4 * PI * x * x * x / x4 * std::cos(xi) * cosx * sinx);
                    bz = ey; by = -ez;
                    ex = a0y * std::sin(xi) * 4 * PI * y * y * y / y4 * cosx * cosx * cosz * cosz * cosy * siny -
                         a0z * std::cos(xi) * 4 * PI * z * z * z / z4 * cosx * cosx * cosy * cosy * cosz * sinz;
                    bx = a0z * std::cos(xi) * 4 * PI * y * y * y / y4 * cosx * cosx * cosz * cosz * cosy * siny +
                         a0y * std::sin(xi) * 4 * PI * z * z * z / z4 * cosx * cosx * cosy * cosy * cosz * sinz;
                } else if (c.sscos == 2) {  // pearl: (sin r / r) transverse (init.cpp:135-150)
                    const double cosx = std::cos(PI * x / 2 / xs), sinx = std::sin(PI * x / 2 / xs);
                    const double r = std::sqrt(y * y + z * z);
                    const double sr = r != 0 ? std::sin(PI * r / c.ysigma) / (PI * r / c.ysigma) : 1.0;
                    ey = a0y * sr * (std::cos(xi) * cosx * cosx - PI / xs * std::sin(xi) * cosx * sinx);
                    ez = a0z * sr * (std::sin(xi) * cosx * cosx + PI / xs * std::cos(xi) * cosx * sinx);
                    bz = ey; by = -ez;
                } else {  // tophat: super-cosine transverse (init.cpp:151-166)
                    const double cosx = std::cos(PI * x / 2 / xs), sinx = std::sin(PI * x / 2 / xs);
                    const double r = std::sqrt(y * y + z * z);
                    const double cy = r <= ys ? std::cos(PI * r * r * r * r / 2 / (ys * ys * ys * ys)) : 0.0;
                    ey = a0y * cy * cy * (std::cos(xi) * cosx * cosx - PI / xs * std::sin(xi) * cosx * sinx);
                    ez = a0z * cy * cy * (std::sin(xi) * cosx * cosx + PI / xs * std::cos(xi) * cosx * sinx);
                    bz = ey; by = -ez;
                }
                if (!c.b_sign) { bx = -bx; by = -by; bz = -bz; }
                const long a = g.at(i, j, k);
                F[0][a] += ex * r0x + ey * y0x + ez * z0x;
                F[1][a] += ex * r0y + ey * y0y + ez * z0y;
                F[2][a] += ex * r0z + ey * y0z + ez * z0z;
                F[3][a] += bx * r0x + by * y0x + bz * z0x;
                F[4][a] += bx * r0y + by * y0y + bz * z0y;
                F[5][a] += bx * r0z + by * y0z + bz * z0z;
            }
}

// f_init_focused with append = true (init.cpp:212-385): a pulse focused to
// the waist sigma0, whose centre (x1, y0, z0) lies at distance L from the
// focus on its axis r0; K is the harmonic (1, or 2 for the second harmonic).
// xi is the phase coordinate along the axis with the wavefront curvature and
// the Gouy phase; slocal the beam radius there.  Inside |xi| < xs and r <
// slocal the envelope is cos^2 (sscos 0, only within the cone r <= 2 s0
// (x1 - x) / xR, outside of which the paraxial fields have unphysical
// wings) or super-cosine^2 in xi (sscos 1), times cos^2 (pi r / 2 slocal);
// E_x and B_x follow from the transverse derivatives of the envelope.  The
// scalar chain up to the envelope tests keeps the reference's operation
// order, so that every cell falls on the same side of each test.
void laser_focused(const Config& c, const Grid3& g, std::vector<double>* F, double a0y, double a0z, double xc,
                   double x1, double y0, double z0, double phase, double phi, double K) {
    const double sign = (x1 <= 0) - (x1 > 0);
    x1 = std::sqrt(x1 * x1 + y0 * y0 + z0 * z0);
    if (x1 == 0) x1 = c.dx;  // the pulse axis needs a direction
    const double sigma0 = c.sigma0;
    const double xR = K * sigma0 * sigma0 / 2;
    const double sigma = sigma0 * std::sqrt(1 + x1 * x1 / xR / xR);
    // the first harmonic's beam radius over this harmonic's at the start
    const double amul = std::sqrt(1 + x1 * x1 / (sigma0 * sigma0 * sigma0 * sigma0 / 4)) /
                        std::sqrt(1 + x1 * x1 / (xR * xR));
    const double xs = c.sscos == 1 ? 0.822 * c.xsigma : c.xsigma * 2 * std::sqrt(2 * PI) / 3;
    const double sn = std::sqrt(((double)3) / 16 - 1 / PI / PI);
    const double s = sigma / 2 / sn, s0 = sigma0 / 2 / sn;
    const double y12 = g.ny * c.dy / 2, z12 = g.nz * c.dz / 2;
    const double r0x = sign * std::sqrt(x1 * x1 - y0 * y0 - z0 * z0) / x1, r0y = -y0 / x1, r0z = -z0 / x1;
    double y0x, y0y, y0z = std::sqrt(r0x * r0x + r0y * r0y);
    if (y0z != 0) { y0x = -r0y / y0z; y0y = r0x / y0z; y0z = 0; }
    else { y0x = 0; y0y = 1; y0z = 0; }
    double z0x = r0y * y0z - r0z * y0y, z0y = r0z * y0x - r0x * y0z, z0z = r0x * y0y - r0y * y0x;
    if (phi != 0) {
        const double cs = std::cos(phi), ss = std::sin(phi);
        const double yx = y0x, yy = y0y, yz = y0z, zx = z0x, zy = z0y, zz = z0z;
        y0x = yx * cs + zx * ss; y0y = yy * cs + zy * ss; y0z = yz * cs + zz * ss;
        z0x = zx * cs - yx * ss; z0y = zy * cs - yy * ss; z0z = zz * cs - yz * ss;
    }
    const double gouy0 = std::atan(x1 / xR);
    const double xs4 = xs * xs * xs * xs;
    for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
            for (int k = 0; k < g.nz; k++) {
                const double X = i * c.dx - xc - c.xtarget, Y = j * c.dy - y12 - y0 - c.ytarget,
                             Z = k * c.dz - z12 - z0 - c.ztarget;
                const double x = r0x * X + r0y * Y + r0z * Z;
                const double r = std::sqrt(X * X + Y * Y + Z * Z - x * x);
                const double xi = x + r * r / 2 * (x - x1) / ((x - x1) * (x - x1) + xR * xR) - std::atan((x - x1) / xR) - gouy0;
                const double w = xi - x1 + gouy0;
                const double slocal = s0 * std::sqrt(1 + w * w / (xR * xR));
                const double alocal = s / slocal * amul;
                if (!(xi > -xs && xi < xs && r < slocal)) continue;
                double ex = 0, ey = 0, ez = 0, bx = 0, by = 0, bz = 0;
                // longitudinal envelope cx = cos(ax), its derivative factor D:
                // d(cx^2)/dxi = -2 D cx sx
                double ax = 0, D = 0;
                bool lit = true;
                if (c.sscos == 1) {
                    ax = PI * xi * xi * xi * xi / 2 / xs4;
                    D = 4 * PI * xi * xi * xi / xs4;
                } else if (-2 * s0 * (x1 - x) / xR <= r && r <= 2 * s0 * (x1 - x) / xR) {
                    ax = PI * xi / 2 / xs;
                    D = PI / xs;
                } else {
                    lit = false;
                }
                if (lit) {
                    const double cx = std::cos(ax), sx = std::sin(ax);
                    const double ar = PI * r / 2 / slocal;
                    const double cr = std::cos(ar), sr = std::sin(ar);
                    const double psi = K * xi + phase, cp = std::cos(psi), sp = std::sin(psi);
                    const double C = cr * cr, cxx = cx * cx, cxs = cx * sx;
                    // the phase-envelope combinations of the field formulas
                    const double P = K * sp * cxx + D * cp * cxs;
                    const double Q = K * cp * cxx - D * sp * cxs;
                    const double Rr = K * cp * cxx + D * sp * cxs;
                    const double Ay = alocal * a0y / K, Az = alocal * a0z / K;
                    ey = Ay * C * Q;
                    ez = -Az * C * P;
                    bz = ey;
                    by = -ez;
                    if (r != 0) {
                        // projections on the polarisation axes, the curvature factor
                        const double Ly = X * y0x + Y * y0y + Z * y0z, Lz = X * z0x + Y * z0y + Z * z0z;
                        const double G = (x - x1) / ((x - x1) * (x - x1) + xR * xR);
                        const double T = cr * sr * PI / slocal / r;
                        ex = Ay * (T * Ly * P - Ly * G * C * Q) - Az * (-T * Lz * Rr - Lz * G * C * P);
                        bx = Ay * (T * Lz * P - Lz * G * C * Q) + Az * (-T * Ly * Rr - Ly * G * C * P);
                    }
                }
                if (!c.b_sign) { bx = -bx; by = -by; bz = -bz; }
                const long a = g.at(i, j, k);
                F[0][a] += ex * r0x + ey * y0x + ez * z0x;
                F[1][a] += ex * r0y + ey * y0y + ez * z0y;
                F[2][a] += ex * r0z + ey * y0z + ez * z0z;
                F[3][a] += bx * r0x + by * y0x + bz * z0x;
                F[4][a] += bx * r0y + by * y0y + bz * z0y;
                F[5][a] += bx * r0z + by * y0z + bz * z0z;
            }
}

struct Parts {
    std::vector<double> x, y, z, ux, uy, uz, g, q;
    void add(double X, double Y, double Z, double UX, double UY, double UZ, double G, double Q) {
        x.push_back(X); y.push_back(Y); z.push_back(Z);
        ux.push_back(UX); uy.push_back(UY); uz.push_back(UZ); g.push_back(G); q.push_back(Q);
    }
    // The order place() leaves the particles in: each is inserted at the head
    // of its cell's list (plist.cpp:22-39), so within a cell the last one
    // created comes first.  qp_load_particles keeps the given order within
    // a cell, so the particles are handed over last first.
    Parts head_order() const {
        Parts r = *this;
        for (auto* v : {&r.x, &r.y, &r.z, &r.ux, &r.uy, &r.uz, &r.g, &r.q}) std::reverse(v->begin(), v->end());
        return r;
    }
};

// fill_cell_by_particles (init.cpp:402-478): a regular in-cell lattice of
// xn*yn*zn particles; thermal momenta drawn like the reference (gamma from
// an exponential by rejection, isotropic direction, boost by the drift);
// a zero drift leaves the direction unrotated (the reference divides by it).
void fill_cell(Parts& P, double cmr, int ci, int cj, int ck, int xn, int yn, int zn, double n, double ux0, double T,
               std::mt19937_64& rng, double dsplmt = 0, double uy0 = 0) {
    std::uniform_real_distribution<double> U(0.0, 1.0);
    const double x0 = 0.5 / xn + dsplmt, y0 = 0.5 / yn, z0 = 0.5 / zn;
    double q0 = 1 / double(xn * yn * zn) * n;
    if (cmr < 0) q0 = -q0;
    for (int ip = 0; ip < xn; ip++)
        for (int jp = 0; jp < yn; jp++)
            for (int kp = 0; kp < zn; kp++) {
                const double X = x0 + ci + double(ip) / xn, Y = y0 + cj + double(jp) / yn, Z = z0 + ck + double(kp) / zn;
                double ux = ux0, uy = uy0, uz = 0;
                if (T != 0 && cmr != 0) {
                    const double u0 = std::fabs(ux0), v0 = u0 / std::sqrt(1 + u0 * u0);
                    double gamma, a, b, cc, r;
                    do { gamma = 1 + U(rng) * 5 * T; } while (U(rng) > std::exp(-(gamma - 1) / T));
                    do {
                        a = 2 * U(rng) - 1; b = 2 * U(rng) - 1; cc = 2 * U(rng) - 1;
                        r = std::sqrt(a * a + b * b + cc * cc);
                    } while (r > 1 || r == 0);
                    a /= r; b /= r; cc /= r;
                    const double vv = std::sqrt(1 - 1 / (gamma * gamma));
                    a *= vv; b *= vv; cc *= vv;
                    b = b * std::sqrt(1 - v0 * v0) / (1 + a * v0);
                    cc = cc * std::sqrt(1 - v0 * v0) / (1 + a * v0);
                    a = (a + v0) / (1 + a * v0);
                    const double gg = 1 / std::sqrt(1 - a * a - b * b - cc * cc);
                    const double sx = ux0 < 0 ? -1.0 : 1.0;
                    ux = sx * a * gg; uy = b * gg; uz = cc * gg;
                }
                const double G = cmr != 0 ? std::sqrt(1 + ux * ux + uy * uy + uz * uz) : std::sqrt(ux * ux + uy * uy + uz * uz);
                P.add(X, Y, Z, ux, uy, uz, G, q0);
            }
}

// film (init.cpp:537-646).  shift: how far the window has moved (x0 of the
// film in window coordinates is x0 - shift); append: fill only the layer
// nx-3 the window just exposed, if the film covers it
// (append_for_moving_window, init.cpp:559-570); profiled: the transverse
// envelope the reference applies when neutral flows are on.
void film(const Config& c, const Grid3& g, const Film& f, Parts& e, Parts* ion, double ion_cmr, Parts* pos,
          std::mt19937_64& rng, double shift = 0, bool append = false, bool profiled = false) {
    int i0 = (int)((f.x0 - shift) / c.dx), i1 = (int)((f.x0 + f.width - shift) / c.dx);
    if (append) {
        i0 = g.nx - 3;
        if (i0 < g.nx - 2 && i1 >= g.nx - 2) i1 = g.nx - 2;
        else i1 = i0;
    } else {
        i0 = std::max(0, std::min(i0, g.nx));
        i1 = std::max(0, std::min(i1, g.nx));
    }
    const double ne_y0 = f.ne_y0 / (1.11485e+13 / c.lambda / c.lambda);
    const double ne_y1 = f.ne_y1 / (1.11485e+13 / c.lambda / c.lambda);
    const double ux0 = f.vx / std::sqrt(1 - f.vx * f.vx);
    const int jy0 = (int)(f.y0 / c.dy), jy1 = (int)(f.y1 / c.dy);
    const double film_ylen = double(jy1 - jy0 - 3);
    for (int i = i0; i < i1; i++)
        for (int j = jy0 + 1; j < jy1 - 1; j++) {
            const double nes_j = ne_y1 * (j - jy0 - 1) / film_ylen + ne_y0 * (jy1 - 2 - j) / film_ylen;
            double nes_run = nes_j;  // the reference scales nes in place along k (init.cpp:583-600)
            for (int k = (int)(f.z0 / c.dz) + 1; k < (int)(f.z1 / c.dz) - 1; k++) {
                if (profiled) {
                    double tmp = (j * c.dy - g.ny * c.dy / 2) / (g.ny * c.dy / 2);
                    tmp = std::cos(0.5 * PI * tmp * tmp * tmp * tmp * tmp);
                    double tr_env = tmp * tmp;
                    tmp = (k * c.dz - g.nz * c.dz / 2) / (g.nz * c.dz / 2);
                    tmp = std::cos(0.5 * PI * tmp * tmp * tmp * tmp * tmp);
                    tr_env *= tmp * tmp;
                    nes_run *= tr_env;
                }
                if (f.grad_y >= 0 && j - jy0 - 1 < f.grad_y / c.dy) nes_run *= (j - jy0 - 1) / (f.grad_y / c.dy);
                if (f.grad_y >= 0 && jy1 - 2 - j < f.grad_y / c.dy) nes_run *= (jy1 - 2 - j) / (f.grad_y / c.dy);
                double nes = nes_run;
                const double fx0 = f.x0 - shift;
                if (f.grad >= 0) {
                    if (!(i >= (int)((fx0 + f.grad) / c.dx))) nes = nes * (i * c.dx - fx0) / f.grad;
                } else {
                    if (!(i >= (int)((fx0 - f.grad) / c.dx))) nes = nes * (1 + (i * c.dx - fx0) / f.grad);
                }
                if (!(nes > 0)) continue;
                fill_cell(e, -1, i, j, k, f.xn, f.yn, f.zn, nes, ux0, f.T, rng);
                if (ion) fill_cell(*ion, ion_cmr, i, j, k, f.xn, f.yn, f.zn, nes, ux0, f.T * ion_cmr, rng);
                if (pos) fill_cell(*pos, 1, i, j, k, f.xn, f.yn, f.zn, nes, ux0, f.T, rng);
            }
        }
}

// add_beam (init.cpp:480-535): a beam of particles of charge sign cmr with
// a parabolic density profile (length 2 xb, radius rb) moving along phib in
// the xy plane, and the fields of an infinitely relativistic beam; cells
// outside [1, n-2) lose their particles (place)
void add_beam(const Config& c, const Grid3& g, std::vector<double>* F, Parts& P, double cmr, double n0, double u0,
              double x0b, std::mt19937_64& rng) {
    const double xb = c.xb, rb = c.rb, y0b = c.y0b, phib = c.phib;
    const double signum = (u0 > 0) - (u0 < 0), type = (cmr > 0) - (cmr < 0);
    for (int i = 0; i < g.nx; i++)
        for (int j = 0; j < g.ny; j++)
            for (int k = 0; k < g.nz; k++) {
                const double phi = std::atan2((j - g.ny / 2) * c.dy - y0b, i * c.dx - x0b);
                const double rr = std::sqrt((i * c.dx - x0b) * (i * c.dx - x0b) +
                                            ((j - g.ny / 2) * c.dy - y0b) * ((j - g.ny / 2) * c.dy - y0b));
                const double x = rr * std::cos(phi - phib), y = rr * std::sin(phi - phib);
                const double z = (k - g.nz / 2) * c.dz;
                const double r = std::sqrt(y * y + z * z);
                if (!(x > -xb && x < xb)) continue;
                double f_ampl;
                if (r < rb) {
                    const double n = n0 * (1 - x * x / (xb * xb)) * (1 - r * r / (rb * rb));
                    if (i > 0 && i < g.nx - 2 && j > 0 && j < g.ny - 2 && k > 0 && k < g.nz - 2)
                        fill_cell(P, cmr, i, j, k, c.xnpic, c.ynpic, c.znpic, n, u0 * std::cos(phib), 0, rng, 0,
                                  u0 * std::sin(phib));
                    f_ampl = 0.5 * n0 * (1 - x * x / (xb * xb)) * (1 - r * r / (2 * rb * rb));
                } else {
                    f_ampl = 0.25 * n0 * (1 - x * x / (xb * xb)) * rb * rb / (r * r);
                }
                const long a = g.at(i, j, k);
                F[0][a] -= type * f_ampl * y * std::sin(phib);
                F[1][a] += type * f_ampl * y * std::cos(phib);
                F[2][a] += type * f_ampl * z;
                F[3][a] += type * signum * f_ampl * z * std::sin(phib);
                F[4][a] -= type * signum * f_ampl * z * std::cos(phib);
                F[5][a] += type * signum * f_ampl * y;
            }
}

// lin_interpolation (low-level.cpp:492-510): 1 without a profile
double lin_interp(double x, const std::vector<double>& xs, const std::vector<double>& vs) {
    if (xs.empty()) return 1.0;
    if (x < xs[0]) return vs[0];
    if (x > xs.back()) return vs.back();
    const size_t i = std::lower_bound(xs.begin(), xs.end(), x) - xs.begin();
    if (i == 0) return vs[0];
    return vs[i - 1] + (vs[i] - vs[i - 1]) * (x - xs[i - 1]) / (xs[i] - xs[i - 1]);
}

// ------------------------------------------------------------- schedule ----
// OutputIterations (parameters.cpp:6-48)
struct Schedule {
    std::vector<int> it;
    std::vector<double> t;
    Schedule(const std::vector<double>& t_end, const std::vector<double>& period, double dt) {
        int prev = -1;
        double t_begin = 0;
        for (size_t i = 0; i < t_end.size(); i++) {
            const int count = (int)((t_end[i] + 0.5 * dt - t_begin) / period[i]) + 1;
            for (int j = 0; j < count; j++) {
                const double time = t_begin + j * period[i];
                const int iter = (int)std::round(time / dt);
                if (iter > prev) { t.push_back(time); it.push_back(iter); prev = iter; }
            }
            t_begin = t_end[i];
        }
        const int last = (int)std::round(t_end.back() / dt);
        if (last > prev) { t.push_back(t_end.back()); it.push_back(last); }
    }
    static std::string suffix(double time) {
        const double v = (int)std::round(time / 2 / PI * 100.) / 100.;
        char b[64];
        snprintf(b, sizeof b, "%g", v);
        return b;
    }
};

// ---------------------------------------------------------------- output ---
// Field slice file (fout.cpp:180-235 and the yz plane writers): for each i
// the xy line at k = nz/2 then the xz line at j = ny/2, then the yz plane at
// i = ix.  Text: one value per line with the default ostream precision.
// values in the slice file's format: text, one per line, or raw doubles
void write_values(const std::string& path, const double* a, size_t n, bool binary) {
    if (binary) {
        std::ofstream f(path, std::ios::out | std::ios::binary);
        f.write((const char*)a, n * sizeof(double));
    } else {
        std::ofstream f(path);
        for (size_t i = 0; i < n; i++) f << a[i] << "\n";
    }
}

void write_slice(const std::string& path, const double* F, const Grid3& g, int ix, bool binary) {
    std::vector<double> a;
    a.reserve((size_t)g.nx * (g.ny + g.nz) + (size_t)g.ny * g.nz);
    for (int i = 0; i < g.nx; i++) {
        for (int j = 0; j < g.ny; j++) a.push_back(F[g.at(i, j, g.nz / 2)]);
        for (int k = 0; k < g.nz; k++) a.push_back(F[g.at(i, g.ny / 2, k)]);
    }
    for (int j = 0; j < g.ny; j++)
        for (int k = 0; k < g.nz; k++) a.push_back(F[g.at(ix, j, k)]);
    if (binary) {
        std::ofstream f(path, std::ios::out | std::ios::binary);
        f.write((const char*)a.data(), a.size() * sizeof(double));
    } else {
        std::ofstream f(path);
        for (double v : a) f << v << "\n";
    }
}

}  // namespace

int main(int argc, char** argv) {
    std::ios::sync_with_stdio(false);
    std::string initial_fields;  // --initial-fields <file>: write the initial E, B and stop
    for (int a = 1; a < argc; a++) {
        if (std::string(argv[a]) == "--initial-fields" && a + 1 < argc) initial_fields = argv[++a];
        else { std::cerr << "usage: qp_driver [--initial-fields <file>] < parsed-input" << std::endl; return 2; }
    }
    Config c;
    try {
        c = parse(read_stream(std::cin));
    } catch (const std::exception& e) {
        std::cerr << "qp_driver: " << e.what() << std::endl;
        return 1;
    }
    Grid3 g{(int)(c.xlength / c.dx), (int)(c.ylength / c.dy), (int)(c.zlength / c.dz)};
    mkdir(c.data_folder.c_str(), 0755);

    // species table: electrons, then ions per film / positrons, then QED
    qp_params p;
    memset(&p, 0, sizeof p);
    p.nx = g.nx; p.ny = g.ny; p.nz = g.nz;
    p.dx = c.dx; p.dy = c.dy; p.dz = c.dz; p.dt = c.dt;
    p.lambda_cm = c.lambda;
    p.solver = c.solver; p.pusher = c.pusher; p.qed = c.qed; p.precision = c.precision;
    p.seed = c.seed;
    int n = 0;
    const int sp_e = n; p.cmr[n++] = -1;
    int sp_pos = -1, sp_ph = -1;
    // ion populations (main.cpp:3250-3325): the distinct mcr of the films
    // (last film first), then of the flows, then of the window's ions; one
    // species each
    std::vector<double> mcrs;
    auto add_mcr = [&](double m) {
        if (std::find(mcrs.begin(), mcrs.end(), m) == mcrs.end()) mcrs.push_back(m);
    };
    if (c.ions == "on" || c.ions == "positrons") {
        for (size_t f = c.films.size(); f-- > 0;) add_mcr(c.films[f].mcr);
        if (c.lflow.n != 0) add_mcr(c.lflow.mcr);
        if (c.rflow.n != 0) add_mcr(c.rflow.mcr);
        if (c.mwindow && !c.mw_auto && c.mwseed_ions) add_mcr(c.mw_mcr);
    }
    std::vector<double> icmr;
    std::vector<int> sp_pop;
    for (double m : mcrs) {
        icmr.push_back(1 / (PROTON_MASS * m));
        sp_pop.push_back(n);
        p.cmr[n++] = icmr.back();
    }
    auto ion_species = [&](double mcr) {
        return (int)(std::find(mcrs.begin(), mcrs.end(), mcr) - mcrs.begin());
    };
    std::vector<int> sp_ion(c.films.size(), -1);
    if (c.ions == "on")
        for (size_t f = 0; f < c.films.size(); f++) sp_ion[f] = sp_pop[ion_species(c.films[f].mcr)];
    if (c.ions == "positrons" || c.qed || (c.beam && c.beam_particles == "p")) { sp_pos = n; p.cmr[n++] = 1; }
    if (c.qed || (c.beam && c.beam_particles == "ph")) { sp_ph = n; p.cmr[n++] = 0; }
    p.n_species = n;

    // initial fields: the default call of init_fields (main.cpp:1186-1189),
    // plus the counter-propagating pulse for phi != 0 (main.cpp:1190-1192)
    std::vector<double> F[6];
    for (auto& f : F) f.assign(g.nc(), 0.0);
    if (c.uniform_b) {
        // f_init_uniformB (init.cpp:387-400)
        for (long a = 0; a < g.nc(); a++) { F[4][a] = c.a0y; F[5][a] = c.a0z; }
    } else if (c.a0y != 0 || c.a0z != 0) {
        // init_fields (main.cpp:1041-1229): the pulse, its
        // counter-propagating copy for phi != 0, or its mirror images; the
        // cos and focused branches place their pulses the same way
        const double A = c.a0y, Z = c.a0z, x0 = c.x0, y0 = c.y00, z0 = c.z00, xl = c.xlength / 2;
        auto split = [](const std::string& s) {
            std::vector<std::string> p(3);
            size_t k = 0;
            for (char ch : s) { if (ch == '&') { if (++k == 3) break; } else p[k] += ch; }
            return p;
        };
        const std::vector<std::string> lp = split(c.lp_reflection), fr = split(c.f_reflection);
        auto sy = [&](int m) { return (1 - 2 * (fr[m] == "y")) * A; };
        auto sz = [&](int m) { return (1 - 2 * (fr[m] == "z")) * Z; };
        auto P = [&](double ay, double az, double xc, double x1, double yy, double zz, double ph) {
            if (c.focused) laser_focused(c, g, F, ay, az, xc, x1, yy, zz, c.phase, ph, 1);
            else laser_cos(c, g, F, ay, az, xc, x1, yy, zz, ph);
        };
        if (c.focused && c.shenergy != 0) {
            // the second harmonic takes the share shenergy of the energy
            const double al = std::sqrt(1 - c.shenergy), be = std::sqrt(c.shenergy);
            laser_focused(c, g, F, A * al, Z * al, xl + x0, x0, y0, z0, c.phase, 0, 1);
            laser_focused(c, g, F, A * be, Z * be, xl + x0, x0, y0, z0, c.shphase, 0, 2);
        } else if (!c.focused && c.phi_rotate != 0) {
            P(A, Z, xl + x0, x0, y0, z0, c.phi_rotate);
        } else {
            P(A, Z, xl + x0, x0, y0, z0, 0);
        }
        if (c.focused || c.phi_rotate == 0) {  // (a rotated cos pulse has no copies)
            if (c.phi != 0) {
                P(A, Z, xl - x0, -x0, -y0, -z0, c.phi);
            } else if (lp[0] == "xy") {
                P(sy(0), sz(0), xl + x0, x0, y0, -z0, 0);
                if (lp[1] == "xz") {
                    P(sy(1), sz(1), xl + x0, x0, -y0, z0, 0);
                    P(sy(1), sz(1), xl + x0, x0, -y0, -z0, 0);
                    if (lp[2] == "yz") {
                        // the reference takes the z sign of the second reflection here
                        P(sy(2), sz(1), -x0 + xl, -x0, y0, z0, 0);
                        P(sy(2), sz(1), -x0 + xl, -x0, y0, -z0, 0);
                        P(sy(2), sz(1), -x0 + xl, -x0, -y0, z0, 0);
                        P(sy(2), sz(1), -x0 + xl, -x0, -y0, -z0, 0);
                    }
                } else if (lp[1] == "yz") {
                    P(sy(1), sz(1), -x0 + xl, -x0, y0, z0, 0);
                    P(sy(1), sz(1), -x0 + xl, -x0, y0, -z0, 0);
                    if (lp[2] == "xz") {
                        P(sy(2), sz(1), -x0 + xl, -x0, -y0, z0, 0);
                        P(sy(2), sz(1), x0 + xl, x0, -y0, z0, 0);
                        P(sy(2), sz(1), -x0 + xl, -x0, -y0, -z0, 0);
                        P(sy(2), sz(1), x0 + xl, x0, -y0, -z0, 0);
                    }
                }
            } else if (lp[0] == "xz") {
                P(sy(0), sz(0), xl + x0, x0, -y0, z0, 0);
                if (lp[1] == "yz") {
                    P(sy(1), sz(1), -x0 + xl, -x0, -y0, z0, 0);
                    P(sy(1), sz(1), -x0 + xl, -x0, y0, z0, 0);
                }
            } else if (lp[0] == "yz") {
                P(sy(0), sz(0), -x0 + xl, -x0, y0, z0, 0);
            }
        }
    }
    // init_beam (main.cpp:1230-1239), after the laser and before the films
    std::mt19937_64 rng(c.seed * 0x9E3779B97F4A7C15ull + 1);
    Parts B;
    int sp_beam = -1;
    if (c.beam) {
        const double n0 = c.Nb * 1.061e-11 / (c.xb * c.rb * c.rb * c.lambda);
        const double x0b = c.xlength - c.x0b;
        if (c.beam_particles == "ph") {
            sp_beam = sp_ph;
            add_beam(c, g, F, B, 0, n0, c.epsb / 0.511, x0b, rng);
        } else {
            const double u0 = ((c.epsb > 0) - (c.epsb < 0)) * std::sqrt(c.epsb * c.epsb / (0.511 * 0.511) - 1);
            sp_beam = c.beam_particles == "p" ? sp_pos : sp_e;
            add_beam(c, g, F, B, c.beam_particles == "p" ? 1 : -1, n0, u0, x0b, rng);
        }
    }
    if (!initial_fields.empty()) {
        std::ofstream o(initial_fields, std::ios::binary);
        for (auto& f : F) o.write(reinterpret_cast<const char*>(f.data()), (std::streamsize)(f.size() * sizeof(double)));
        return o ? 0 : 1;
    }
    qp_handle* h = nullptr;
    if (qp_create(&p, &h) != QP_OK) {
        std::cerr << "qp_driver: " << qp_last_error(nullptr) << std::endl;
        return 1;
    }
    int r = qp_load_fields(h, F[0].data(), F[1].data(), F[2].data(), F[3].data(), F[4].data(), F[5].data());
    if (r == QP_OK) r = qp_init_boundaries(h);
    // films, loaded species by species (cell order is sorted inside the library)
    Parts E;
    std::vector<Parts> I(mcrs.size());
    Parts Pz;
    const bool profiled = c.lflow.n != 0 || c.rflow.n != 0;
    for (size_t f = c.films.size(); f-- > 0;) {
        const int pi = sp_ion[f] >= 0 ? ion_species(c.films[f].mcr) : -1;
        film(c, g, c.films[f], E, pi >= 0 ? &I[pi] : nullptr, pi >= 0 ? icmr[pi] : 0,
             c.ions == "positrons" ? &Pz : nullptr, rng, 0, false, profiled);
    }
    auto load = [&](int s, const Parts& P0) {
        if (r != QP_OK || P0.x.empty()) return;
        const Parts P = P0.head_order();
        r = qp_load_particles(h, s, (int64_t)P.x.size(), P.x.data(), P.y.data(), P.z.data(), P.ux.data(),
                              P.uy.data(), P.uz.data(), P.g.data(), P.q.data(), nullptr);
    };
    if (sp_beam >= 0) load(sp_beam, B);
    load(sp_e, E);
    if (c.ions == "on")
        for (size_t k = 0; k < mcrs.size(); k++) load(sp_pop[k], I[k]);
    if (sp_pos >= 0) load(sp_pos, Pz);
    if (r != QP_OK) {
        std::cerr << "qp_driver: " << qp_last_error(h) << std::endl;
        qp_destroy(h);
        return 1;
    }

    // catching: erased particles recorded on the device, drained every step
    // into the host list the reference keeps (deleted_particles), cumulative
    // deleted energies per class (update_energy_deleted)
    struct Caught { int32_t sp; double q, x, y, z, ux, uy, uz, g, chi; };
    std::vector<Caught> caught;
    double e_del = 0, p_del = 0, ph_del = 0;
    std::vector<double> i_del(icmr.size(), 0.0);
    int i_particle = 0, i_particle_p = 0, i_particle_ph = 0, i_particle_i = 0;
    if (r == QP_OK && c.n_tracks > 0) r = qp_set_tracking(h, 1);
    if (r == QP_OK && c.ordered_current) r = qp_set_ordered_current(h, 1);
    std::ofstream fED;
    if (r == QP_OK && (c.catching || c.dump_photons)) {
        int64_t total = 0, np = 0;
        for (int s2 = 0; s2 < n; s2++) { qp_count_particles(h, s2, &np); total += np; }
        const int64_t cap = std::max<int64_t>(total, 1 << 16);
        if (c.catching) {
            r = qp_set_erased_tracking(h, 1);
            if (r == QP_OK) r = qp_set_catching(h, 1, cap);
        }
        if (r == QP_OK && c.dump_photons) r = qp_set_dump_photons(h, 1, cap);
        fED.open(c.data_folder + "/energy_deleted");
    }
    if (r != QP_OK) {
        std::cerr << "qp_driver: " << qp_last_error(h) << std::endl;
        qp_destroy(h);
        return 1;
    }

    // log in the reference's name/value layout (main.cpp:3611-3785 subset)
    {
        std::ofstream L(c.data_folder + "/log");
        L << "dx\n" << c.dx / 2 / PI << "\ndy\n" << c.dy / 2 / PI << "\ndz\n" << c.dz / 2 / PI << "\ndt\n" << c.dt / 2 / PI << "\n";
        L << "nx\n" << g.nx << "\nny\n" << g.ny << "\nnz\n" << g.nz << "\n";
        L << "lambda\n" << c.lambda << "\nne\n" << c.ne << "\n";
        for (size_t i = 0; i < c.t_end.size(); i++)
            L << "t_end\n" << c.t_end[i] / 2 / PI << "\noutput_period\n" << c.output_period[i] / 2 / PI << "\n";
        L << "xsigma\n" << c.xsigma / 2 / PI << "\nysigma\n" << c.ysigma / 2 / PI << "\nzsigma\n" << c.zsigma / 2 / PI << "\n";
        L << "x0fout\n" << c.xlength / 2 / 2 / PI << "\n";
        L << "a0y\n" << c.a0y << "\na0z\n" << c.a0z << "\n";
        L << "mwindow\n" << (c.mwindow ? "on" : "off") << "\n";
        L << "e_components_for_output\n" << c.e_out << "\nb_components_for_output\n" << c.b_out << "\n";
        L << "n_ion_populations\n" << icmr.size() << "\n";
        for (double v : icmr) L << "icmr\n" << v << "\n";
        L << "xnpic\n" << c.xnpic << "\nynpic\n" << c.ynpic << "\nznpic\n" << c.znpic << "\n";
        L << "particles_for_output\n" << c.particles_for_output << "\n";
        L << "enthp\n" << c.enthp << "\n";
        L << "n_sr\n1\n$\n";
        L << "catching\noff\ndump_photons\n" << (c.dump_photons ? "on" : "off") << "\nqed\n" << (c.qed ? "on" : "off") << "\n";
        L << "balancing\noff\noutput_mode\n" << (c.binary ? 1 : 0) << "\n";
        L << "#------------------------------\n";
        L << "polarization = " << c.polarization << "\n";
        L << "solver = " << (c.solver == QP_SOLVER_FDTD ? "fdtd" : c.solver == QP_SOLVER_NDFX ? "ndfx" : "five_point") << "\n";
        L << "pusher = " << (c.pusher == QP_PUSHER_BORIS ? "boris" : "vay") << "\n";
        L << "precision = " << (c.precision == QP_PREC_MIXED ? "mixed" : "fp64") << "\n";
        L << "pmerging\n" << c.pmerging << "\ncrpc\n" << c.crpc << "\n";
        L << "catching\n" << (c.catching ? "on" : "off") << "\n";
    }

    // particle merging: evaluate_merging_condition (main.cpp:1691-1748) after
    // each step, pmerging before the next (main.cpp:2321-2322); ppd is kept
    // per class (electrons, positrons, photons, ion populations) and mapped
    // onto the species table
    const int n_ion = (int)icmr.size();
    const double crnp = c.crpc * c.xlength * c.ylength * c.zlength / (c.dx * c.dy * c.dz);
    bool merge_now = false;
    std::vector<double> ppd(3 + n_ion, 0.0), ppd_sp(QP_MAX_SPECIES, 0.0);
    auto evaluate_merging = [&](const qp_diag& d) {
        merge_now = false;
        if (c.pmerging == "ti") {
            int64_t nq = d.N_qp_e + d.N_qp_p + d.N_qp_g;
            for (int i = 0; i < n_ion; i++) nq += d.N_qp_i[i];
            if (nq > (3 + n_ion) * crnp) {
                merge_now = true;
                ppd[0] = (nq - (3 + n_ion) * crnp) / nq;
                for (int s2 = 0; s2 < QP_MAX_SPECIES; s2++) ppd_sp[s2] = ppd[0];
            }
        } else if (c.pmerging == "nl") {
            std::vector<int64_t> nq = {d.N_qp_e, d.N_qp_p, d.N_qp_g};
            for (int i = 0; i < n_ion; i++) nq.push_back(d.N_qp_i[i]);
            for (size_t k = 0; k < nq.size(); k++) {
                ppd[k] = nq[k] > crnp ? (nq[k] - crnp) / nq[k] : 0.0;
                if (nq[k] > crnp) merge_now = true;
            }
            ppd_sp.assign(QP_MAX_SPECIES, 0.0);
            ppd_sp[sp_e] = ppd[0];
            if (sp_pos >= 0) ppd_sp[sp_pos] = ppd[1];
            if (sp_ph >= 0) ppd_sp[sp_ph] = ppd[2];
            for (size_t k = 0; k < sp_pop.size(); k++) ppd_sp[sp_pop[k]] = ppd[3 + k];
        }
    };

    // time loop (main.cpp:2319-2432)
    Schedule sch(c.t_end, c.output_period, c.dt);
    std::ofstream fN(c.data_folder + "/N"), fE(c.data_folder + "/energy");
    size_t out_i = 0;
    std::vector<double> slices(12 * ((size_t)g.nx * (g.ny + g.nz) + (size_t)g.ny * g.nz));
    // the yz plane of the field and density files: x = xlength - x0fout
    // (get_xindex_in_sr, main.cpp:144-147)
    const int ix = std::min(g.nx - 1, std::max(0, (int)((c.xlength - c.x0fout) / c.dx)));
    // moving window state (main.cpp:122, 2665-2679)
    int nmw = 1;
    const double t_add_mw = c.t_add_mw != 0 ? c.t_add_mw : sch.it.back() * c.dt;
    std::ofstream fMW;
    if (c.mwindow) fMW.open(c.data_folder + "/mwcoordinate");
    // add_moving_window_particles (main.cpp:1750-1883): the layer nx-3 the
    // window exposed gets uniform plasma (mwseed, density ne) and the part of
    // every film it now covers
    auto add_window_particles = [&](int l) -> int {
        if (!((l + 1) * c.dt < t_add_mw)) return QP_OK;
        Parts Em, Pm;
        std::vector<Parts> Im(mcrs.size());
        // mwseed / mwseed_ions: density ne times the x profile at the window's
        // offset and the radial profile of each (j, k) line (main.cpp:1756-1821)
        const double n = c.ne / (1.11485e+13 / c.lambda / c.lambda) *  // 1 / k0^2 (main.cpp:2602)
                         lin_interp((nmw - 1) * c.dx, c.prof_x, c.prof_xv);
        auto seed_layer = [&](Parts& P, double cmr) {
            for (int j = 0; j < (int)(c.ylength / c.dy); j++)
                for (int k = 0; k < (int)(c.zlength / c.dz); k++) {
                    const double yr = j * c.dy - c.ylength / 2.0, zr = k * c.dz - c.zlength / 2.0;
                    const double mod = lin_interp(std::sqrt(zr * zr + yr * yr), c.prof_r, c.prof_rv);
                    if (mod != 0.0) fill_cell(P, cmr, g.nx - 3, j, k, c.xnpic, c.ynpic, c.znpic, n * mod, 0, 0, rng);
                }
        };
        if (c.mwseed) seed_layer(Em, -1);
        const int mw_pop = c.mwseed_ions ? ion_species(c.mw_mcr) : -1;
        if (mw_pop >= 0 && mw_pop < (int)mcrs.size()) seed_layer(Im[mw_pop], icmr[mw_pop]);
        for (size_t f = c.films.size(); f-- > 0;) {
            const int pi = sp_ion[f] >= 0 ? ion_species(c.films[f].mcr) : -1;
            film(c, g, c.films[f], Em, pi >= 0 ? &Im[pi] : nullptr, pi >= 0 ? icmr[pi] : 0,
                 c.ions == "positrons" ? &Pm : nullptr, rng, nmw * c.dx, true);
        }
        int rr = QP_OK;
        auto put = [&](int sp, const Parts& P0) {
            if (rr != QP_OK || P0.x.empty()) return;
            const Parts P = P0.head_order();
            rr = qp_load_particles(h, sp, (int64_t)P.x.size(), P.x.data(), P.y.data(), P.z.data(), P.ux.data(),
                                   P.uy.data(), P.uz.data(), P.g.data(), P.q.data(), nullptr);
        };
        put(sp_e, Em);
        for (size_t k = 0; k < mcrs.size(); k++) put(sp_pop[k], Im[k]);
        if (sp_pos >= 0) put(sp_pos, Pm);
        return rr;
    };
    // start_tracking (main.cpp:1516-1612, the line mode): the first particle
    // of each requested kind in every distinct cell along the line from
    // (xtr1, ytr1, ztr1) to (xtr2, ytr2, ztr2) gets the next track number
    const int nm = 4;  // nx_ich / 2 (main.cpp:2232-2233)
    bool tracking = false;
    auto start_tracking = [&]() -> int {
        if (c.xtr1 < 0 || c.xtr2 < 0 || c.ytr1 < 0 || c.ytr2 < 0 || c.ztr1 < 0 || c.ztr2 < 0 || c.xtr1 >= c.xlength ||
            c.xtr2 >= c.xlength || c.ytr1 >= c.ylength || c.ytr2 >= c.ylength || c.ztr1 >= c.zlength ||
            c.ztr2 >= c.zlength) {
            std::cout << "Error - tracks outside of compulational domain" << std::endl;
            return QP_OK;
        }
        std::vector<int64_t> cells;
        if (!c.tr_volume) {
            int x1 = -1, y1 = 0, z1 = 0;
            for (int i = 0; i < c.n_tracks; i++) {
                const int x2 = (int)((c.xtr1 + (c.xtr2 - c.xtr1) * i / c.n_tracks) / c.dx);
                const int y2 = (int)((c.ytr1 + (c.ytr2 - c.ytr1) * i / c.n_tracks) / c.dy);
                const int z2 = (int)((c.ztr1 + (c.ztr2 - c.ztr1) * i / c.n_tracks) / c.dz);
                if (x2 != x1 || y2 != y1 || z2 != z1) {
                    x1 = x2; y1 = y2; z1 = z2;
                    cells.push_back(((int64_t)x2 * g.ny + y2) * g.nz + z2);
                }
            }
        } else {
            // volume: a uniformly drawn cell of the box per track (the reference draws with rand())
            std::uniform_real_distribution<double> U(0.0, 1.0);
            for (int i = 0; i < c.n_tracks; i++) {
                const int x1 = (int)((c.xtr1 + (c.xtr2 - c.xtr1) * U(rng)) / c.dx);
                const int y1 = (int)((c.ytr1 + (c.ytr2 - c.ytr1) * U(rng)) / c.dy);
                const int z1 = (int)((c.ztr1 + (c.ztr2 - c.ztr1) * U(rng)) / c.dz);
                cells.push_back(((int64_t)x1 * g.ny + y1) * g.nz + z1);
            }
        }
        // kinds in the reference's order per cell: e, p, g, then every ion population
        std::vector<int> kinds;
        if (c.particles_to_track.find('e') != std::string::npos) kinds.push_back(sp_e);
        if (c.particles_to_track.find('p') != std::string::npos && sp_pos >= 0) kinds.push_back(sp_pos);
        if (c.particles_to_track.find('g') != std::string::npos && sp_ph >= 0) kinds.push_back(sp_ph);
        if (c.particles_to_track.find('i') != std::string::npos)
            for (int s2 : sp_pop) kinds.push_back(s2);
        std::vector<std::vector<int64_t>> first(kinds.size(), std::vector<int64_t>(cells.size()));
        for (size_t k = 0; k < kinds.size(); k++) {
            const int rr = qp_first_in_cells(h, kinds[k], (int64_t)cells.size(), cells.data(), first[k].data());
            if (rr != QP_OK) return rr;
        }
        std::vector<std::vector<int64_t>> pos(kinds.size()), num(kinds.size());
        int64_t trn = 1;
        for (size_t cc = 0; cc < cells.size(); cc++)
            for (size_t k = 0; k < kinds.size(); k++)
                if (first[k][cc] >= 0) {
                    // a cell drawn again renumbers its first particle, as the reference overwrites trn
                    auto it = std::find(pos[k].begin(), pos[k].end(), first[k][cc]);
                    if (it != pos[k].end()) num[k][it - pos[k].begin()] = trn++;
                    else { pos[k].push_back(first[k][cc]); num[k].push_back(trn++); }
                }
        for (size_t k = 0; k < kinds.size(); k++) {
            const int rr = qp_set_track_numbers(h, kinds[k], (int64_t)pos[k].size(), pos[k].data(), num[k].data());
            if (rr != QP_OK) return rr;
        }
        tracking = true;
        return QP_OK;
    };
    // fout_tracks (fout.cpp:706-734): one file per tracked particle, 9 values per step
    auto fout_tracks = [&](double a) -> int {
        for (int s2 = 0; s2 < n; s2++) {
            int64_t m = 0;
            int rr = qp_get_tracked(h, s2, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                                    nullptr, nullptr, &m);
            if (rr != QP_OK) return rr;
            if (m == 0) continue;
            std::vector<int64_t> tn(m);
            std::vector<double> t9[9];
            for (auto& v2 : t9) v2.resize(m);
            rr = qp_get_tracked(h, s2, m, tn.data(), t9[0].data(), t9[1].data(), t9[2].data(), t9[3].data(),
                                t9[4].data(), t9[5].data(), t9[6].data(), t9[7].data(), t9[8].data(), &m);
            if (rr != QP_OK) return rr;
            char cm[32];
            snprintf(cm, sizeof cm, "%g", p.cmr[s2]);
            for (int64_t t = 0; t < m; t++) {
                if (!(t9[0][t] >= nm && t9[0][t] < g.nx - nm)) continue;
                std::ofstream T(c.data_folder + "/track_" + cm + "_" + std::to_string(tn[t]), std::ios::app);
                T << t9[7][t] << '\n' << t9[0][t] * c.dx / 2 / PI + a << '\n' << t9[1][t] * c.dy / 2 / PI << '\n'
                  << t9[2][t] * c.dz / 2 / PI << '\n' << t9[3][t] << '\n' << t9[4][t] << '\n' << t9[5][t] << '\n'
                  << t9[6][t] << '\n' << t9[8][t] << '\n';
            }
        }
        return QP_OK;
    };
    // add_neutral_flow_particles (main.cpp:1837-1880): when the flow has
    // advanced one cell, a layer of plasma with a transverse envelope enters
    // at i = 2..3 (from the left) or nx-4..nx-3 (from the right); the entry
    // offset follows the reference's xrflow for both faces
    double xlflow = 1, xrflow = 1;
    auto add_flow = [&](int dir, const Flow& fl) -> int {
        double& xflow = dir > 0 ? xlflow : xrflow;
        int rr = QP_OK;
        if (xflow >= 1) {
            xflow -= 1;
            const double nn = fl.n / c.xnpic;
            const double u = dir * fl.v / std::sqrt(1 - fl.v * fl.v);
            Parts Ef, If;
            const int pi = c.ions == "on" ? ion_species(fl.mcr) : -1;
            for (int j = 0; j < (int)(c.ylength / c.dy); j++)
                for (int k = 0; k < (int)(c.zlength / c.dz); k++)
                    for (int ii = 0; ii < c.xnpic; ii++) {
                        double x0 = xrflow - float(ii) / c.xnpic;
                        int ci;
                        if (x0 >= 0) ci = dir > 0 ? 3 : g.nx - 4;
                        else { ci = dir > 0 ? 2 : g.nx - 3; x0 += 1; }
                        double tmp = (j * c.dy - c.ylength / 2) / (c.ylength / 2);
                        tmp = std::cos(0.5 * PI * tmp * tmp * tmp * tmp * tmp);
                        double tr_env = tmp * tmp;
                        tmp = (k * c.dz - c.zlength / 2) / (c.zlength / 2);
                        tmp = std::cos(0.5 * PI * tmp * tmp * tmp * tmp * tmp);
                        tr_env *= tmp * tmp;
                        const double ds = (dir > 0 ? x0 : 1 - x0) - 0.5;
                        fill_cell(Ef, -1, ci, j, k, 1, c.ynpic, c.znpic, nn * tr_env, u, fl.T, rng, ds);
                        if (pi >= 0)
                            fill_cell(If, icmr[pi], ci, j, k, 1, c.ynpic, c.znpic, nn * tr_env, u,
                                      fl.T / (PROTON_MASS * fl.mcr), rng, ds);
                    }
            // place(): only particles inside the region stay (plist.cpp:22-39)
            auto keep_inside = [&](Parts& P) {
                Parts Q;
                for (size_t t = 0; t < P.x.size(); t++) {
                    const int i = (int)P.x[t], j = (int)P.y[t], k = (int)P.z[t];
                    if (i > 0 && i < g.nx - 2 && j > 0 && j < g.ny - 2 && k > 0 && k < g.nz - 2)
                        Q.add(P.x[t], P.y[t], P.z[t], P.ux[t], P.uy[t], P.uz[t], P.g[t], P.q[t]);
                }
                return Q;
            };
            const Parts Eq = keep_inside(Ef).head_order(), Iq = keep_inside(If).head_order();
            if (!Eq.x.empty())
                rr = qp_load_particles(h, sp_e, (int64_t)Eq.x.size(), Eq.x.data(), Eq.y.data(), Eq.z.data(),
                                       Eq.ux.data(), Eq.uy.data(), Eq.uz.data(), Eq.g.data(), Eq.q.data(), nullptr);
            if (rr == QP_OK && pi >= 0 && !Iq.x.empty())
                rr = qp_load_particles(h, sp_pop[pi], (int64_t)Iq.x.size(), Iq.x.data(), Iq.y.data(), Iq.z.data(),
                                       Iq.ux.data(), Iq.uy.data(), Iq.uz.data(), Iq.g.data(), Iq.q.data(), nullptr);
        }
        xflow += c.dt * fl.v / c.dx;
        return rr;
    };
    for (int l = 0; l <= sch.it.back(); l++) {
        qp_diag d;
        if (merge_now && qp_pmerging(h, c.pmerging == "ti" ? QP_MERGE_TI : QP_MERGE_NL, ppd_sp.data()) != QP_OK) {
            std::cerr << "qp_driver: merging before step " << l << ": " << qp_last_error(h) << std::endl;
            qp_destroy(h);
            return 1;
        }
        if (qp_step(h, 1, c.external_bz, &d) != QP_OK) {
            std::cerr << "qp_driver: step " << l << ": " << qp_last_error(h) << std::endl;
            qp_destroy(h);
            return 1;
        }
        fN << d.N_e << '\t' << d.N_p << '\t' << d.N_ph << std::endl;  // write_N, main.cpp:160-170
        fE << d.energy_f << '\t' << d.energy_e << '\t' << d.energy_p << '\t' << d.energy_ph;  // write_energy
        for (int m = 0; m < d.n_ion; m++) fE << '\t' << d.ienergy[m];
        fE << std::endl;
        if (c.n_tracks > 0 && tracking && fout_tracks(nmw * c.dx / 2 / PI) != QP_OK) {
            std::cerr << "qp_driver: tracks at step " << l << ": " << qp_last_error(h) << std::endl;
            qp_destroy(h);
            return 1;
        }
        // check_moving_window (main.cpp:1953-1978, 2333-2336): mode on moves
        // with mwspeed; mode auto moves when the front slice's max E^2 + B^2
        // exceeds mwtolerance times the box's
        bool mw_now = false;
        if (c.mwindow && !c.mw_auto) {
            mw_now = (l + 1) * c.dt * c.mwspeed > nmw * c.dx;
        } else if (c.mw_auto) {
            double max_w = 0, front = 0;
            if (qp_max_w(h, 0, g.nx, &max_w) != QP_OK || qp_max_w(h, g.nx - nm - 2, g.nx - nm, &front) != QP_OK) {
                std::cerr << "qp_driver: max_w after step " << l << ": " << qp_last_error(h) << std::endl;
                qp_destroy(h);
                return 1;
            }
            const double ratio = max_w > 0 ? front / max_w : 0.0;
            mw_now = ratio > c.mwtolerance;
        }
        if (mw_now) {
            if (qp_moving_window(h) != QP_OK) {
                std::cerr << "qp_driver: moving window after step " << l << ": " << qp_last_error(h) << std::endl;
                qp_destroy(h);
                return 1;
            }
            nmw++;
        }
        if (c.mwindow) fMW << ((nmw - 1) * c.dx / 2 / PI) << std::endl;  // write_mwcoordinate
        if (c.catching || c.dump_photons) {
            // drain the device records (deletion order inside a species)
            int64_t m = 0, dropped = 0;
            qp_get_caught(h, 0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                          nullptr, &m, &dropped);
            if (m > 0) {
                std::vector<int32_t> sp(m);
                std::vector<double> a[9];
                for (auto& v2 : a) v2.resize(m);
                qp_get_caught(h, m, sp.data(), a[0].data(), a[1].data(), a[2].data(), a[3].data(), a[4].data(),
                              a[5].data(), a[6].data(), a[7].data(), a[8].data(), &m, &dropped);
                for (int64_t t = 0; t < m; t++)
                    caught.push_back({sp[t], a[7][t], a[0][t], a[1][t], a[2][t], a[3][t], a[4][t], a[5][t], a[6][t], a[8][t]});
            }
            if (dropped > 0) std::cerr << "qp_driver: step " << l << ": " << dropped << " erased particles not recorded" << std::endl;
            // write_energy_deleted (main.cpp:353-367): cumulative, per class
            e_del += d.energy_erased_sp[sp_e];
            if (sp_pos >= 0) p_del += d.energy_erased_sp[sp_pos];
            if (sp_ph >= 0) ph_del += d.energy_erased_sp[sp_ph];
            for (size_t k = 0; k < sp_pop.size(); k++) i_del[k] += d.energy_erased_sp[sp_pop[k]];
            fED << e_del << '\t' << p_del << '\t' << ph_del;
            for (double v2 : i_del) fED << '\t' << v2;
            fED << std::endl;
        }
        evaluate_merging(d);
        if (out_i < sch.it.size() && l == sch.it[out_i]) {
            const std::string sfx = Schedule::suffix(sch.t[out_i]);
            // the output slices come from the device (qp_dump_field_slices)
            const size_t per = (size_t)g.nx * (g.ny + g.nz) + (size_t)g.ny * g.nz;
            qp_dump_field_slices(h, ix, slices.data());
            const size_t NC = (size_t)g.nc();
            // currents (write_density with scale_j, main.cpp:2346-2349,
            // 369-415): J scaled by dx / dt, as spatial_region::scale_j does
            for (int a = 0; a < 3; a++) {
                if (!c.write_j[a]) continue;
                std::vector<double> jv(slices.data() + (6 + a) * per, slices.data() + (7 + a) * per);
                for (double& x2 : jv) x2 *= c.dx / c.dt;
                write_values(c.data_folder + "/j" + std::string(1, "xyz"[a]) + sfx, jv.data(), per, c.binary);
            }
            // every species in traversal order (each species' particles in the
            // order of the reference's cell lists)
            struct SpDump { std::vector<double> x, y, z, ux, uy, uz, g, q, chi; };
            auto dump = [&](int si) {
                SpDump D;
                if (si < 0) return D;
                int64_t np = 0;
                qp_count_particles(h, si, &np);
                for (auto* vv : {&D.x, &D.y, &D.z, &D.ux, &D.uy, &D.uz, &D.g, &D.q, &D.chi}) vv->resize(np);
                if (np) qp_dump_particles(h, si, np, D.x.data(), D.y.data(), D.z.data(), D.ux.data(), D.uy.data(),
                                          D.uz.data(), D.g.data(), D.q.data(), D.chi.data(), nullptr);
                return D;
            };
            const SpDump De_ = dump(sp_e), Dp_ = dump(c.write_p ? sp_pos : -1), Dph_ = dump(c.write_ph ? sp_ph : -1);
            std::vector<SpDump> Di_(sp_pop.size());
            for (size_t m = 0; m < sp_pop.size(); m++) Di_[m] = dump(sp_pop[m]);
            // densities (compute_rho + rhodeposition, fout.cpp:7-40,
            // deposition.cpp:358-429): cloud-in-cell charge of the particles
            // in is_inside cells, in the reference's term order
            auto cic = [&](const SpDump& D, std::vector<double>& rho) {
                for (size_t t = 0; t < D.x.size(); t++) {
                    const int i = (int)std::floor(D.x[t]), j = (int)std::floor(D.y[t]), k = (int)std::floor(D.z[t]);
                    if (!(i > 0 && i < g.nx - 2 && j > 0 && j < g.ny - 2 && k > 0 && k < g.nz - 2)) continue;
                    const double xa = D.x[t] - i, xb = 1 - xa, ya = D.y[t] - j, yb = 1 - ya, za = D.z[t] - k, zb = 1 - za;
                    const double qq = D.q[t];
                    rho[g.at(i, j, k)] += qq * xb * yb * zb;
                    rho[g.at(i + 1, j, k)] += qq * xa * yb * zb;
                    rho[g.at(i, j + 1, k)] += qq * xb * ya * zb;
                    rho[g.at(i, j, k + 1)] += qq * xb * yb * za;
                    rho[g.at(i + 1, j + 1, k)] += qq * xa * ya * zb;
                    rho[g.at(i + 1, j, k + 1)] += qq * xa * yb * za;
                    rho[g.at(i, j + 1, k + 1)] += qq * xb * ya * za;
                    rho[g.at(i + 1, j + 1, k + 1)] += qq * xa * ya * za;
                }
            };
            {
                // write_density(true, write_p, write_ph, "rho", "rho_p", "rho_ph", true)
                const SpDump* ds[3] = {&De_, &Dp_, &Dph_};
                const bool wr[3] = {true, c.write_p, c.write_ph};
                const char* names[3] = {"rho", "rho_p", "rho_ph"};
                for (int w = 0; w < 3; w++) {
                    if (!wr[w]) continue;
                    std::vector<double> rho(NC, 0.0);
                    cic(*ds[w], rho);
                    write_slice(c.data_folder + "/" + names[w] + sfx, rho.data(), g, ix, c.binary);
                }
                // ion densities irho_<cmr>_ (main.cpp:440-470, fout.cpp:662-704)
                if (c.ions == "on" || c.ions == "positrons")
                    for (size_t m = 0; m < sp_pop.size(); m++) {
                        std::vector<double> rho(NC, 0.0);
                        cic(Di_[m], rho);
                        char b2[32];
                        snprintf(b2, sizeof b2, "%g", icmr[m]);
                        write_slice(c.data_folder + "/irho_" + b2 + "_" + sfx, rho.data(), g, ix, c.binary);
                    }
            }
            // spectra and phase space (write_spectrum_phasespace,
            // main.cpp:478-743): dN/deps in 1/MeV from the charge per energy
            // bin; 9 values (q, x y z in lambda, ux uy uz, g, chi) of every
            // particle after which a class's counter passes its enthp
            {
                const double vol = 1.11485e13 * c.lambda * c.dx * c.dy * c.dz / (8 * PI * PI * PI);
                auto ps_put = [&](std::ofstream& o, const SpDump& D, size_t t) {
                    o << D.q[t] << "\n" << c.dx * D.x[t] / (2 * PI) << "\n" << c.dy * D.y[t] / (2 * PI) << "\n"
                      << c.dz * D.z[t] / (2 * PI) << "\n" << D.ux[t] << "\n" << D.uy[t] << "\n" << D.uz[t] << "\n"
                      << D.g[t] << "\n" << D.chi[t] << "\n";
                };
                std::ofstream PSe(c.data_folder + "/phasespace" + sfx), PSp(c.data_folder + "/phasespace_p" + sfx),
                    PSph(c.data_folder + "/phasespace_ph" + sfx);
                std::vector<double> spec(std::max(c.neps, 0), 0.0), spec_p(std::max(c.neps_p, 0), 0.0),
                    spec_ph(std::max(c.neps_ph, 0), 0.0);
                for (size_t t = 0; t < De_.x.size(); t++) {
                    const int ie = (int)((De_.g[t] - 1) * 0.511 / c.deps);
                    if (ie > -1 && ie < c.neps) spec[ie] = spec[ie] - De_.q[t];
                    if (++i_particle > c.enthp) { i_particle = 0; ps_put(PSe, De_, t); }
                }
                for (size_t t = 0; t < Dp_.x.size(); t++) {
                    const int ie = (int)((Dp_.g[t] - 1) * 0.511 / c.deps_p);
                    if (ie > -1 && ie < c.neps_p) spec_p[ie] = spec_p[ie] + Dp_.q[t];
                    if (++i_particle_p > c.enthp_p) { i_particle_p = 0; ps_put(PSp, Dp_, t); }
                }
                for (size_t t = 0; t < Dph_.x.size(); t++) {
                    const int ie = (int)(Dph_.g[t] * 0.511 / c.deps_ph);
                    if (ie > -1 && ie < c.neps_ph) spec_ph[ie] = spec_ph[ie] + Dph_.q[t];
                    if (++i_particle_ph > c.enthp_ph) { i_particle_ph = 0; ps_put(PSph, Dph_, t); }
                }
                std::vector<std::vector<double>> spec_i(sp_pop.size(), std::vector<double>(std::max(c.neps_i, 0), 0.0));
                for (size_t m = 0; m < sp_pop.size(); m++) {
                    char b2[32];
                    snprintf(b2, sizeof b2, "%g", icmr[m]);
                    std::ofstream PSi(c.data_folder + "/phasespace_" + b2 + "_" + sfx);
                    const SpDump& D = Di_[m];
                    for (size_t t = 0; t < D.x.size(); t++) {
                        const int ie = (int)((D.g[t] - 1) * 0.511 * PROTON_MASS / c.deps_i);
                        if (ie > -1 && ie < c.neps_i) spec_i[m][ie] += D.q[t];
                        if (++i_particle_i > c.enthp_i) { i_particle_i = 0; ps_put(PSi, D, t); }
                    }
                }
                std::ofstream S(c.data_folder + "/spectrum" + sfx), Sp(c.data_folder + "/spectrum_p" + sfx),
                    Sph(c.data_folder + "/spectrum_ph" + sfx);
                for (double& x2 : spec) { x2 = x2 * (vol / c.deps); S << x2 << "\n"; }
                if (c.write_p)
                    for (double& x2 : spec_p) { x2 = x2 * (vol / c.deps_p); Sp << x2 << "\n"; }
                if (c.write_ph)
                    for (double& x2 : spec_ph) { x2 = x2 * (vol / c.deps_ph); Sph << x2 << "\n"; }
                for (size_t m = 0; m < sp_pop.size(); m++) {
                    char b2[32];
                    snprintf(b2, sizeof b2, "%g", icmr[m]);
                    std::ofstream Si(c.data_folder + "/spectrum_" + b2 + "_" + sfx);
                    const double norm_i = vol / (icmr[m] * c.deps_i);
                    for (double& x2 : spec_i[m]) { x2 = x2 * norm_i; Si << x2 << "\n"; }
                }
            }
            if (c.catching || c.dump_photons) {
                // write_deleted_particles (main.cpp:189-345): 9 values per
                // written particle, the reference's every-n-th counters, and
                // the deleted photons' spectrum; the list is then cleared
                // main.cpp:3392-3395
                const std::string& pf = c.particles_for_output;
                const bool write_p = pf == "ep" || pf == "epph";
                const bool write_ph = pf == "eph" || pf == "epph";
                std::ofstream De(c.data_folder + "/deleted" + sfx), Dp(c.data_folder + "/deleted_p" + sfx),
                    Dph(c.data_folder + "/deleted_ph" + sfx);
                std::vector<std::ofstream> Di(icmr.size());
                for (size_t m = 0; m < icmr.size(); m++) {
                    char b[32];
                    snprintf(b, sizeof b, "%g", icmr[m]);
                    Di[m].open(c.data_folder + "/deleted_" + b + "_" + sfx);
                }
                std::vector<double> spec(std::max(c.neps_ph, 0), 0.0);
                auto put = [&](std::ofstream& o, const Caught& k) {
                    o << k.q << '\n' << c.dx * k.x / (2 * PI) << '\n' << c.dy * k.y / (2 * PI) << '\n'
                      << c.dz * k.z / (2 * PI) << '\n' << k.ux << '\n' << k.uy << '\n' << k.uz << '\n' << k.g << '\n'
                      << k.chi << '\n';
                };
                for (const Caught& k : caught) {
                    if (k.sp == sp_e) {
                        if (++i_particle > c.enthp) { i_particle = 0; put(De, k); }
                    } else if (write_p && k.sp == sp_pos) {
                        if (++i_particle_p > c.enthp_p) { i_particle_ph = 0; put(Dp, k); }
                    } else if (write_ph && k.sp == sp_ph) {
                        const int ie = c.deps_ph > 0 ? (int)(k.g * 0.511 / c.deps_ph) : -1;
                        if (ie > -1 && ie < c.neps_ph) spec[ie] += k.q;
                        if (++i_particle_ph > c.enthp_ph) { i_particle_ph = 0; put(Dph, k); }
                    } else {
                        for (size_t m = 0; m < sp_pop.size(); m++)
                            if (k.sp == sp_pop[m]) {
                                if (++i_particle_i > c.enthp_i) { i_particle_i = 0; put(Di[m], k); }
                                break;
                            }
                    }
                }
                caught.clear();
                if (write_ph && c.deps_ph > 0) {
                    std::ofstream S(c.data_folder + "/spectrum_deleted_ph" + sfx);
                    const double norm = 1.11485e13 * c.lambda * c.dx * c.dy * c.dz / (8 * PI * PI * PI) / c.deps_ph;
                    for (double v2 : spec) S << v2 * norm << '\n';
                }
            }
            // layer weights (write_layer_weights, main.cpp:997-1039): ny*nz
            // plus balancing_particle_weight per particle of the layer
            {
                std::vector<int64_t> cnt(g.nx, 0);
                qp_layer_counts(h, cnt.data());
                std::ofstream Wt(c.data_folder + "/weights" + sfx);
                // the reference gathers region 0's layers up to nx - nx_ich/2
                // whatever n_sr is (main.cpp:1005-1008): with one region its
                // last 4 layers stay 0
                for (int i = 0; i < g.nx; i++) {
                    double wgt = (double)g.ny * g.nz;
                    for (int64_t u = 0; u < cnt[i]; u++) wgt += c.balancing_particle_weight;
                    Wt << (i < g.nx - 4 ? wgt : 0.0) << "\n";
                }
            }
            // fields (write_fields, main.cpp:745-995): the chosen E and B
            // components, then w = E^2 + B^2 and inv = E^2 - B^2 from E and
            // the B average at the slice nodes (e_to_particle / b_to_particle at
            // integer positions, fout.cpp:437-561), always as text
            const char* en[3] = {"ex", "ey", "ez"};
            const char* bn[3] = {"bx", "by", "bz"};
            for (int a = 0; a < 3; a++) {
                const char comp = "xyz"[a];
                if (c.e_out.find(comp) != std::string::npos)
                    write_values(c.data_folder + "/" + en[a] + sfx, slices.data() + a * per, per, c.binary);
                if (c.b_out.find(comp) != std::string::npos)
                    write_values(c.data_folder + "/" + bn[a] + sfx, slices.data() + (3 + a) * per, per, c.binary);
            }
            {
                // the yz plane of w / inv one layer lower when it is the last
                std::vector<double> plane_lo;
                if (ix == g.nx - 1) {
                    plane_lo.resize(12 * per);
                    qp_dump_field_slices(h, ix - 1, plane_lo.data());
                }
                auto val = [&](const std::vector<double>& src, int comp, size_t at) { return src[comp * per + at]; };
                const size_t yz0 = (size_t)g.nx * (g.ny + g.nz);
                std::ofstream Wf(c.data_folder + "/w" + sfx), If(c.data_folder + "/inv" + sfx);
                auto put = [&](const std::vector<double>& src, size_t at) {
                    const double ex = val(src, 0, at), ey = val(src, 1, at), ez = val(src, 2, at);
                    const double bx = val(src, 9, at), by = val(src, 10, at), bz = val(src, 11, at);
                    Wf << ex * ex + ey * ey + ez * ez + bx * bx + by * by + bz * bz << "\n";
                    If << ex * ex + ey * ey + ez * ez - bx * bx - by * by - bz * bz << "\n";
                };
                for (int i = 0; i < g.nx; i++) {
                    const int ii = i == g.nx - 1 ? i - 1 : i;  // the last region's last layer
                    const size_t row = (size_t)ii * (g.ny + g.nz);
                    for (int j = 0; j < g.ny; j++) put(slices, row + (j == g.ny - 1 ? j - 1 : j));
                    for (int k = 0; k < g.nz; k++) put(slices, row + g.ny + (k == g.nz - 1 ? k - 1 : k));
                }
                const std::vector<double>& src = ix == g.nx - 1 ? plane_lo : slices;
                for (int j = 0; j < g.ny; j++)
                    for (int k = 0; k < g.nz; k++) {
                        const int jj = j == g.ny - 1 ? j - 1 : j, kk = k == g.nz - 1 ? k - 1 : k;
                        put(src, yz0 + (size_t)jj * g.nz + kk);
                    }
            }
            out_i++;
        }
        if (c.n_tracks > 0 && !c.particles_to_track.empty() && l == (int)(c.tr_start / c.dt) &&
            start_tracking() != QP_OK) {
            std::cerr << "qp_driver: start_tracking: " << qp_last_error(h) << std::endl;
            qp_destroy(h);
            return 1;
        }
        if (mw_now && add_window_particles(l) != QP_OK) {
            std::cerr << "qp_driver: window plasma after step " << l << ": " << qp_last_error(h) << std::endl;
            qp_destroy(h);
            return 1;
        }
        if ((c.lflow.n != 0 && add_flow(1, c.lflow) != QP_OK) || (c.rflow.n != 0 && add_flow(-1, c.rflow) != QP_OK)) {
            std::cerr << "qp_driver: neutral flow after step " << l << ": " << qp_last_error(h) << std::endl;
            qp_destroy(h);
            return 1;
        }
    }
    qp_destroy(h);
    return 0;
}
