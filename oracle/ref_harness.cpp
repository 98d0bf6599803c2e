// ref_harness.cpp -- drives the UNMODIFIED reference sources (compiled from the
// reference tree by oracle/Makefile into oracle/_ref/) on one rank through the
// single-rank MPI stand-in in oracle/ref_shim/mpi.h.
//
// TEST INFRASTRUCTURE ONLY: pins the oracle restatement (tests/test_oracle_golden.py,
// tests/golden/make_golden.py) and times the reference CPU path for
// bench.py --impl reference.  It replaces Driver::run (src/driver.cpp:3-72):
// parameters come from the command line instead of input.xml, and the
// primitive field comes from a raw file (halo'd AoS doubles) instead of
// testcases::*.
//
// usage: ref_harness MODE key=value ... (see parse below)
//   MODE rhs   : stage-1 prologue (time_scheme.cpp:124,133-135) then the selected
//                operators into a zeroed R; writes R (halo'd AoS) to out=
//   MODE step  : steps= calls of TimeScheme::step; writes W then U (halo'd AoS)
//                to out=, and the per-step dt to out=.dt
//   MODE dt    : TimeScheme::set_dt on the input W; prints the dt
//   MODE bench : steps= timed TimeScheme::step calls after warmup= untimed ones on
//                a synthetic shear layer (in=shear, the default), Taylor-Green
//                vortex (in=tgv) or a raw file; prints one JSON line
//   MODE ic    : case= one of the test cases Driver::set_initial_condition
//                dispatches (src/driver.cpp:107-141), set by the reference's own
//                testcases.cpp on the zero-initialised Domain; writes W (halo'd AoS)
//                to out= (pins the B200 driver's initial conditions)
//   MODE dropin: (built with NS_WITH_B200) steps= steps of the same state three
//                ways: the reference TimeScheme with its own operators, the
//                reference TimeScheme with the B200 operators plugged in through
//                ns_b200_adapters.hpp, and the B200 GpuTimeScheme; prints the
//                relative L2 differences of W per field as JSON
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "communicator.hpp"
#include "convection_schemes/weno-5.hpp"
#include "convection_schemes/weno-5cw.hpp"
#include "decomposition.hpp"
#include "diffusion_schemes/centered_diffusion.hpp"
#include "domain.hpp"
#include "grid.hpp"
#include "params.hpp"
#include "testcases.hpp"
#include "time_scheme.hpp" // also brings eq_of_state.hpp, whose include guard (EqOfState_hh vs EqOfSTate_hh) admits one inclusion only
#ifdef NS_WITH_B200
#include "ns_b200_adapters.hpp"
#endif

static std::map<std::string, std::string> kv;

static std::string S(const char* k, const char* d) {
    auto it = kv.find(k);
    return it == kv.end() ? std::string(d) : it->second;
}
static double D(const char* k, double d) {
    auto it = kv.find(k);
    return it == kv.end() ? d : atof(it->second.c_str());
}
static int I(const char* k, int d) {
    auto it = kv.find(k);
    return it == kv.end() ? d : atoi(it->second.c_str());
}

// SplitMix64 (Steele, Lea, Flood 2014) for the synthetic timing field
static unsigned long long sm_state;
static double sm_uniform() {
    unsigned long long z = (sm_state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static void shear_layer(Array4d& W, const Params& p) {
    const double pi = 3.14159265358979323846;
    const double dx = p.Lx / p.nx, dy = p.Ly / p.ny;
    const double delta = 0.05 * 2.0 * pi, M = 0.5;
    sm_state = 1;
    for (int i = 0; i < p.nx; i++)
        for (int j = 0; j < p.ny; j++)
            for (int k = 0; k < p.nz; k++) {
                double x = dx * 0.5 + i * dx, y = dy * 0.5 + j * dy;
                double y1 = 0.5 * pi, y2 = 1.5 * pi;
                double u = std::tanh((y - y1) / delta) - std::tanh((y - y2) / delta) - 1.0;
                double g = std::exp(-(y - y1) * (y - y1) / (delta * delta)) +
                           std::exp(-(y - y2) * (y - y2) / (delta * delta));
                double nv = 1e-3 * (2.0 * sm_uniform() - 1.0);
                double nw = 1e-3 * (2.0 * sm_uniform() - 1.0);
                W(i + 3, j + 3, k + 3, 0) = 1.0;
                W(i + 3, j + 3, k + 3, 1) = 1.0 / (p.gamma * M * M);
                W(i + 3, j + 3, k + 3, 2) = u;
                W(i + 3, j + 3, k + 3, 3) = 0.05 * std::sin(x) * g + nv;
                W(i + 3, j + 3, k + 3, 4) = nw;
            }
}

// Compressible Taylor-Green vortex on [0,2pi]^3 (M = 0.1) with seeded velocity
// noise 1e-4, the same field as 3dnssolver_b200/workloads.py taylor_green
// (SplitMix64 stream 5, three draws per cell in i-j-k order)
static void taylor_green(Array4d& W, const Params& p) {
    const double dx = p.Lx / p.nx, dy = p.Ly / p.ny, dz = p.Lz / p.nz, M = 0.1;
    sm_state = 5;
    for (int i = 0; i < p.nx; i++)
        for (int j = 0; j < p.ny; j++)
            for (int k = 0; k < p.nz; k++) {
                double x = dx * 0.5 + i * dx, y = dy * 0.5 + j * dy, z = dz * 0.5 + k * dz;
                double n0 = 1e-4 * (2.0 * sm_uniform() - 1.0);
                double n1 = 1e-4 * (2.0 * sm_uniform() - 1.0);
                double n2 = 1e-4 * (2.0 * sm_uniform() - 1.0);
                W(i + 3, j + 3, k + 3, 0) = 1.0;
                W(i + 3, j + 3, k + 3, 1) = 1.0 / (p.gamma * M * M) +
                                            (std::cos(2 * x) + std::cos(2 * y)) * (std::cos(2 * z) + 2.0) / 16.0;
                W(i + 3, j + 3, k + 3, 2) = std::sin(x) * std::cos(y) * std::cos(z) + n0;
                W(i + 3, j + 3, k + 3, 3) = -std::cos(x) * std::sin(y) * std::cos(z) + n1;
                W(i + 3, j + 3, k + 3, 4) = n2;
            }
}

int main(int argc, char** argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: ref_harness rhs|step|dt|bench key=value...\n");
        return 2;
    }
    std::string mode = argv[1];
    for (int a = 2; a < argc; a++) {
        const char* e = strchr(argv[a], '=');
        if (!e) continue;
        kv[std::string(argv[a], e - argv[a])] = std::string(e + 1);
    }
    MPI_Init(NULL, NULL);
    Params p;
    p.dim = I("dim", 3);
    p.nx = I("nx", 16);
    p.ny = I("ny", 16);
    p.nz = I("nz", 16);
    p.nproc_x = p.nproc_y = p.nproc_z = 1;
    p.Lx = D("Lx", 1.0);
    p.Ly = D("Ly", 1.0);
    p.Lz = D("Lz", 1.0);
    p.mu = D("mu", 1e-3);
    p.Pr = D("Pr", 0.72);
    p.gamma = D("gamma", 1.4);
    p.CFL_max = D("cfl", 0.5);
    p.end_t = 1.0;
    p.io_interval = 1;
    int conv = I("conv", 1);   // 0 none, 1 weno5, 2 weno5 characteristic
    int diff = I("diff", 1);   // 0 none, 1 centered
    p.convection_scheme = conv ? "Weno" : "none";
    p.convection_scheme_order = 5;
    p.convection_in_characteristic_space = (conv == 2);
    p.weight_type = I("weights", 0) ? "Borges" : "Shu";
    p.diffusion_scheme = diff ? "Centered" : "none";
    p.diffusion_scheme_order = I("order", 2);
    const char* names[3][2] = {{"West", "East"}, {"North", "South"}, {"Back", "Front"}};
    const char* keys[3] = {"bcx", "bcy", "bcz"};
    for (int a = 0; a < 3; a++) {
        std::string t = I(keys[a], 0) ? "Neumann" : "Periodic";
        p.boundary_conditions[names[a][0]] = t;
        p.boundary_conditions[names[a][1]] = t;
    }

    Decomposition dec(p);
    Grid grid(p, dec);
    Communicator comm(dec);
    Domain domain(p, dec);
    Array4d& W = domain.get_NS_primitive_array();
    Array4d& U = domain.get_NS_conservative_array();
    const size_t nall = W.NX() * W.NY() * W.NZ() * W.NQ();

    if (mode == "ic") {
        const std::string c = S("case", "sod_x");
        p.testcase = c;
        if (c == "sod_x") testcases::sod_xdir(domain, grid, p);
        else if (c == "sod_y") testcases::sod_ydir(domain, grid, p);
        else if (c == "sod_z") testcases::sod_zdir(domain, grid, p);
        else if (c == "case3") testcases::case3(domain, grid, p);
        else if (c == "case4") testcases::case4(domain, grid, p);
        else if (c == "case6") testcases::case6(domain, grid, p);
        else if (c == "case12") testcases::case12(domain, grid, p);
        else if (c == "case15") testcases::case15(domain, grid, p);
        else if (c == "case17") testcases::case17(domain, grid, p);
        else if (c == "shear_xy") testcases::shear_layer_xy(domain, grid, p);
        else if (c == "shear_3d") testcases::shear_layer_3d(domain, grid, p);
        else {
            fprintf(stderr, "unknown case %s\n", c.c_str());
            return 2;
        }
        FILE* f = fopen(S("out", "ic.bin").c_str(), "wb");
        if (!f || fwrite(&W(0, 0, 0, 0), sizeof(double), nall, f) != nall) return 1;
        fclose(f);
        MPI_Finalize();
        return 0;
    }

    std::string in = S("in", "");
    if (in == "tgv") {
        taylor_green(W, p);
    } else if (!in.empty() && in != "shear") {
        FILE* f = fopen(in.c_str(), "rb");
        if (!f || fread(&W(0, 0, 0, 0), sizeof(double), nall, f) != nall) {
            fprintf(stderr, "cannot read %s\n", in.c_str());
            return 1;
        }
        fclose(f);
    } else {
        shear_layer(W, p);
    }

    // Driver::create_convection_operator / create_diffusion_operator (src/driver.cpp:74-105)
    ConvectionScheme* cs;
    if (conv == 2)
        cs = new Weno5cw("Weno-5cw", p.gamma, p.weight_type);
    else if (conv == 1)
        cs = new Weno5("Weno-5cw", p.gamma, p.weight_type);
    else
        cs = new ConvectionScheme("null", p.gamma);
    DiffusionScheme* ds;
    if (diff)
        ds = new CenteredDiffusion("Centered", p.gamma, p.mu, p.Pr, p.diffusion_scheme_order);
    else
        ds = new DiffusionScheme();
    TimeScheme ts(p);
    std::string out = S("out", "");

    if (mode == "rhs") {
        int terms = I("terms", 3);
        EqOfState eos(p.gamma);
        eos.primitive_to_conservative(W, U);
        domain.apply_boundary_conditions(U);
        comm.communicate(U);
        eos.conservative_to_primitive(U, W);
        Array4d R(W.get_dimensions());
        if (terms & 1) cs->solve(grid, W, U, R);
        if (terms & 2) ds->solve(grid, comm, W, R);
        FILE* f = fopen(out.c_str(), "wb");
        fwrite(&R(0, 0, 0, 0), sizeof(double), nall, f);
        if (I("dump_state", 0)) {
            fwrite(&W(0, 0, 0, 0), sizeof(double), nall, f);
            fwrite(&U(0, 0, 0, 0), sizeof(double), nall, f);
        }
        fclose(f);
    } else if (mode == "step") {
        int steps = I("steps", 1);
        std::vector<double> dts;
        for (int s = 0; s < steps; s++) {
            ts.step(domain, grid, comm, cs, ds);
            dts.push_back(ts.get_dt());
        }
        FILE* f = fopen(out.c_str(), "wb");
        fwrite(&W(0, 0, 0, 0), sizeof(double), nall, f);
        fwrite(&U(0, 0, 0, 0), sizeof(double), nall, f);
        fclose(f);
        f = fopen((out + ".dt").c_str(), "wb");
        fwrite(dts.data(), sizeof(double), dts.size(), f);
        fclose(f);
    } else if (mode == "dt") {
        // set_dt is private; one step's dt is the dt of the input state
        ts.step(domain, grid, comm, cs, ds);
        printf("%.17g\n", ts.get_dt());
    } else if (mode == "bench") {
        int warm = I("warmup", 1), steps = I("steps", 2);
        for (int s = 0; s < warm; s++) ts.step(domain, grid, comm, cs, ds);
        auto t0 = std::chrono::steady_clock::now();
        for (int s = 0; s < steps; s++) ts.step(domain, grid, comm, cs, ds);
        auto t1 = std::chrono::steady_clock::now();
        double sec = std::chrono::duration<double>(t1 - t0).count();
        double cells = (double)p.nx * p.ny * p.nz;
        printf("{\"seconds\": %.6f, \"steps\": %d, \"cell_updates_per_s\": %.6e, \"dt\": %.17g}\n",
               sec, steps, cells * 3.0 * steps / sec, ts.get_dt());
    } else if (mode == "dropin") {
#ifdef NS_WITH_B200
        int steps = I("steps", 3);
        Domain dB(p, dec), dC(p, dec);
        Array4d& WB = dB.get_NS_primitive_array();
        Array4d& WC = dC.get_NS_primitive_array();
        memcpy(&WB(0, 0, 0, 0), &W(0, 0, 0, 0), nall * sizeof(double));
        memcpy(&WC(0, 0, 0, 0), &W(0, 0, 0, 0), nall * sizeof(double));
        ns_b200::Context gctx(p);
        ns_b200::GpuConvection gconv(gctx, p.gamma);
        ns_b200::GpuDiffusion gdiff(gctx, p);
        ConvectionScheme* gc = conv ? (ConvectionScheme*)&gconv : cs;
        DiffusionScheme* gd = diff ? (DiffusionScheme*)&gdiff : ds;
        TimeScheme tsB(p);
        ns_b200::GpuTimeScheme tsC(gctx);
        double dtA = 0, dtB = 0, dtC = 0;
        for (int s = 0; s < steps; s++) {
            ts.step(domain, grid, comm, cs, ds);
            tsB.step(dB, grid, comm, gc, gd);
            tsC.step(dC, grid, comm, gc, gd);
            dtA = ts.get_dt(); dtB = tsB.get_dt(); dtC = tsC.get_dt();
        }
        auto rel = [&](const Array4d& X, int q) {
            double num = 0, den = 0;
            for (size_t i = W.i_begin(); i < W.i_end(); i++)
                for (size_t j = W.j_begin(); j < W.j_end(); j++)
                    for (size_t k = W.k_begin(); k < W.k_end(); k++) {
                        double a = X(i, j, k, q), b = W(i, j, k, q);
                        num += (a - b) * (a - b);
                        den += b * b;
                    }
            return den > 0 ? sqrt(num / den) : sqrt(num);
        };
        printf("{\"steps\": %d, \"dt\": [%.17g, %.17g, %.17g], \"operators\": [", steps, dtA, dtB, dtC);
        for (int q = 0; q < 5; q++) printf("%s%.6e", q ? ", " : "", rel(WB, q));
        printf("], \"time_scheme\": [");
        for (int q = 0; q < 5; q++) printf("%s%.6e", q ? ", " : "", rel(WC, q));
        printf("]}\n");
#else
        fprintf(stderr, "built without NS_WITH_B200\n");
        return 2;
#endif
    } else {
        fprintf(stderr, "unknown mode %s\n", mode.c_str());
        return 2;
    }
    delete cs;
    delete ds;
    MPI_Finalize();
    return 0;
}
