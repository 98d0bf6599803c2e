// ns_b200_driver -- the reference's executable (src/main.cpp, src/driver.cpp)
// on the B200 path: reads the same input.xml (src/io/reader.cpp), checks it
// like Params::sanity_check (src/params.cpp:3-147), sets the named initial
// condition (src/testcases.cpp), and runs TimeScheme::step until EndT through
// the C ABI of ns_b200.h with the state resident on the GPU.
//
//   ns_b200_driver [--input input.xml] [--precision fp64|fp32] [--results DIR]
//                  [--max-steps N] [--restart FILE] [--check] [--dump-ic FILE]
//
// Output (FileFormat Binary, and in place of Hdf5, which this build does not
// link): every OutputInterval steps and at the end, DIR/fields_<iter>_p_0.dat
// in the layout of BinaryWriter::write_fields (src/io/io_binary.cpp:35-73:
// interior cells in i-j-k order, rho p u v w as doubles per cell) with
// DIR/fields_<iter>_p_0.time ("time iter") beside it, and DIR/mesh_p_0.dat
// (BinaryWriter::write_mesh, io_binary.cpp:3-32).  A fields file with its
// .time file is a checkpoint: --restart continues from it (the reference
// writes but cannot restart).
//
// Exit status: 0 done, 1 invalid input (the reference's std::exit(1)), 2 bad
// command line, 3 library/device error, 4 I/O error.
#include <cerrno>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "ns_b200.h"

namespace {

// ---------------------------------------------------------------------------
// a small XML reader: elements, text, comments, the declaration; attributes
// are skipped (the input file has none)

struct XNode {
    std::string name, text;
    std::vector<XNode> kids;
    const XNode* child(const std::string& n) const {
        for (const XNode& k : kids)
            if (k.name == n) return &k;
        return nullptr;
    }
};

struct XmlParser {
    const std::string& s;
    size_t i = 0;
    std::string err;
    explicit XmlParser(const std::string& src) : s(src) {}

    bool starts(const char* t) const { return s.compare(i, strlen(t), t) == 0; }
    bool skip_to(const char* t) {
        size_t j = s.find(t, i);
        if (j == std::string::npos) return false;
        i = j + strlen(t);
        return true;
    }
    void skip_misc() {  // whitespace, comments, declarations
        for (;;) {
            while (i < s.size() && isspace((unsigned char)s[i])) i++;
            if (starts("<?")) { if (!skip_to("?>")) return; continue; }
            if (starts("<!--")) { if (!skip_to("-->")) return; continue; }
            if (starts("<!")) { if (!skip_to(">")) return; continue; }
            return;
        }
    }
    static std::string unescape(const std::string& t) {
        static const std::pair<const char*, char> ent[] = {
            {"&lt;", '<'}, {"&gt;", '>'}, {"&amp;", '&'}, {"&quot;", '"'}, {"&apos;", '\''}};
        std::string o;
        for (size_t k = 0; k < t.size();) {
            bool hit = false;
            if (t[k] == '&')
                for (const auto& e : ent)
                    if (t.compare(k, strlen(e.first), e.first) == 0) {
                        o += e.second;
                        k += strlen(e.first);
                        hit = true;
                        break;
                    }
            if (!hit) o += t[k++];
        }
        return o;
    }
    bool element(XNode& n) {
        if (!starts("<")) { err = "expected an element"; return false; }
        i++;
        size_t b = i;
        while (i < s.size() && !isspace((unsigned char)s[i]) && s[i] != '>' && s[i] != '/') i++;
        n.name = s.substr(b, i - b);
        if (n.name.empty()) { err = "empty element name"; return false; }
        size_t close = s.find('>', i);
        if (close == std::string::npos) { err = "unterminated <" + n.name; return false; }
        bool selfclose = close > 0 && s[close - 1] == '/';
        i = close + 1;
        if (selfclose) return true;
        for (;;) {
            if (i >= s.size()) { err = "unterminated <" + n.name + ">"; return false; }
            if (starts("<!--")) { if (!skip_to("-->")) { err = "unterminated comment"; return false; } continue; }
            if (starts("</")) {
                i += 2;
                size_t e = s.find('>', i);
                if (e == std::string::npos) { err = "unterminated </" + n.name; return false; }
                std::string nm = s.substr(i, e - i);
                while (!nm.empty() && isspace((unsigned char)nm.back())) nm.pop_back();
                if (nm != n.name) { err = "</" + nm + "> closes <" + n.name + ">"; return false; }
                i = e + 1;
                return true;
            }
            if (starts("<")) {
                n.kids.emplace_back();
                if (!element(n.kids.back())) return false;
                continue;
            }
            size_t e = s.find('<', i);
            if (e == std::string::npos) e = s.size();
            n.text += unescape(s.substr(i, e - i));
            i = e;
        }
    }
    bool document(XNode& root) {
        skip_misc();
        if (!element(root)) return false;
        skip_misc();
        return true;
    }
};

std::string trim(const std::string& t) {
    size_t b = 0, e = t.size();
    while (b < e && isspace((unsigned char)t[b])) b++;
    while (e > b && isspace((unsigned char)t[e - 1])) e--;
    return t.substr(b, e - b);
}

// ---------------------------------------------------------------------------
// Params (src/params.hpp) as read by Reader::read_input_file (reader.cpp:3-172)

struct InputError {
    std::string what;
};

struct Params {
    int dim = 0, io_interval = 0, nx = 0, ny = 0, nz = 0, nproc_x = 1, nproc_y = 1, nproc_z = 1;
    double Lx = 0, Ly = 0, Lz = 0, mu = 0, Pr = 0, gamma = 0, CFL_max = 0, end_t = 0;
    std::string testcase, riemann_solver, convection_scheme, weight_type, diffusion_scheme,
        output_file_format;
    int convection_scheme_order = 0, convection_in_characteristic_space = 0, diffusion_scheme_order = 0;
    std::map<std::string, std::string> boundary_conditions;
};

const XNode& section(const XNode& root, const char* name) {
    const XNode* e = root.child(name);
    if (!e) throw InputError{name};
    return *e;
}
std::string text_of(const XNode& parent, const char* name) {
    const XNode* e = parent.child(name);
    if (!e) throw InputError{name};
    return trim(e->text);
}
void read(const XNode& parent, const char* name, int& v) {
    std::string t = text_of(parent, name);
    char* end = nullptr;
    long x = strtol(t.c_str(), &end, 10);
    if (t.empty() || *end) throw InputError{std::string(name) + " (not an integer: '" + t + "')"};
    v = (int)x;
}
void read(const XNode& parent, const char* name, double& v) {
    std::string t = text_of(parent, name);
    char* end = nullptr;
    double x = strtod(t.c_str(), &end);
    if (t.empty() || *end) throw InputError{std::string(name) + " (not a number: '" + t + "')"};
    v = x;
}
void read(const XNode& parent, const char* name, std::string& v) { v = text_of(parent, name); }

Params read_input(const XNode& root) {
    if (root.name != "Input") throw InputError{"Input (first element)"};
    Params p;
    const XNode& g = section(root, "Geometry");
    read(g, "Dim", p.dim);
    read(g, "Lx", p.Lx);
    read(g, "Ly", p.Ly);
    read(g, "Lz", p.Lz);
    const XNode& gr = section(root, "Grid");
    read(gr, "Nx", p.nx);
    read(gr, "Ny", p.ny);
    read(gr, "Nz", p.nz);
    const XNode& f = section(root, "FluidProperties");
    read(f, "Mu", p.mu);
    read(f, "Pr", p.Pr);
    read(f, "Gamma", p.gamma);
    const XNode& t = section(root, "Time");
    read(t, "EndT", p.end_t);
    read(t, "CFLmax", p.CFL_max);
    const XNode& o = section(root, "OutputProperties");
    read(o, "OutputInterval", p.io_interval);
    read(o, "FileFormat", p.output_file_format);
    read(section(root, "InitialConditions"), "Case", p.testcase);
    const XNode& bc = section(root, "BoundaryConditions");
    for (const char* side : {"West", "East", "North", "South", "Front", "Back"}) {
        std::string v;
        read(bc, side, v);
        p.boundary_conditions[side] = v;
    }
    const XNode& ns = section(root, "NumericalSchemes");
    const XNode& cs = section(ns, "ConvectionScheme");
    read(cs, "Scheme", p.convection_scheme);
    if (p.convection_scheme == "Weno") {
        read(cs, "WeightType", p.weight_type);
        read(cs, "RiemannSolver", p.riemann_solver);
    }
    read(cs, "CharacteristicSpace", p.convection_in_characteristic_space);
    read(cs, "Order", p.convection_scheme_order);
    const XNode& ds = section(ns, "DiffusionScheme");
    read(ds, "Scheme", p.diffusion_scheme);
    read(ds, "Order", p.diffusion_scheme_order);
    const XNode& dd = section(root, "DomainDecomposition");
    read(dd, "NprocX", p.nproc_x);
    read(dd, "NprocY", p.nproc_y);
    read(dd, "NprocZ", p.nproc_z);
    return p;
}

template <typename T>
bool one_of(const T& v, std::initializer_list<T> set) {
    for (const T& x : set)
        if (x == v) return true;
    return false;
}

// Params::sanity_check (params.cpp:3-147): prints the choices and rejects
// invalid ones; returns an empty string when valid
std::string sanity_check(const Params& p, bool verbose) {
    std::ostringstream out;
    auto fail = [&](const std::string& m) { return m + " Exiting."; };
    if (!one_of<std::string>(p.testcase, {"random", "sod_x", "sod_y", "sod_z", "case3", "case4", "case6",
                                          "case12", "case15", "case17", "shear_xy", "jet", "rank", "shear_3d"}))
        return fail("Testcase: " + p.testcase + " is not valid.");
    out << "Running test case: " << p.testcase << "\n";
    if (!one_of<std::string>(p.convection_scheme, {"Weno", "Centered", "none"}))
        return fail("Convection scheme: " + p.convection_scheme + " is not valid.");
    out << " Using convection scheme: " << p.convection_scheme << "\n";
    if (p.convection_scheme == "Weno") {
        if (!one_of<std::string>(p.weight_type, {"Shu", "Borges"}))
            return fail("Weight type: " + p.weight_type + " is not valid.");
        out << " With weight type: " << p.weight_type << "\n";
        if (p.convection_scheme_order != 5)
            return fail("Convection scheme order: " + std::to_string(p.convection_scheme_order) + " is not valid.");
    } else if (!one_of(p.convection_scheme_order, {2, 4, 6})) {
        return fail("Convection scheme order: " + std::to_string(p.convection_scheme_order) + " is not valid.");
    }
    out << " Convection scheme order: " << p.convection_scheme_order << "\n";
    out << " Convection in characteristic space? yes/no (0/1): " << p.convection_in_characteristic_space << "\n";
    if (!one_of<std::string>(p.diffusion_scheme, {"Centered", "Shen", "none"}))
        return fail("Diffusion scheme: " + p.diffusion_scheme + " is not valid.");
    out << " Using diffusion scheme: " << p.diffusion_scheme << "\n";
    if (!one_of(p.diffusion_scheme_order, {2, 4, 6}))
        return fail("Diffusion scheme order: " + std::to_string(p.diffusion_scheme_order) + " is not valid.");
    out << " Diffusion scheme order: " << p.diffusion_scheme_order << "\n";
    out << "Boundary conditions: \n";
    for (const auto& bc : p.boundary_conditions) {
        if (!one_of<std::string>(bc.second, {"Periodic", "Neumann", "Inflow"}))
            return fail("Boundary condition: " + bc.second + " is not valid (at " + bc.first + ").");
        out << bc.first << " " << bc.second << "\n";
    }
    if (!one_of<std::string>(p.output_file_format, {"Hdf5", "Binary"}))
        return fail("Output file format: " + p.output_file_format + " is not valid.");
    out << " Output file format: " << p.output_file_format << "\n";
    if (verbose) std::cout << out.str();
    return "";
}

// What the reference accepts but cannot run on one rank: reported instead of
// the crash or NaN state the reference would produce.
std::string b200_limits(const Params& p) {
    // Driver::set_initial_condition (driver.cpp:107-141) sets no state for these
    if (one_of<std::string>(p.testcase, {"random", "jet", "rank"}))
        return "test case " + p.testcase + " sets no initial state in the reference's Driver";
    if (p.convection_scheme == "Weno" && p.riemann_solver != "LaxFriedrichs")
        return "RiemannSolver " + p.riemann_solver + " (only LaxFriedrichs exists)";
    // Decomposition takes periodicity from West/South/Front (decomposition.cpp:145-161);
    // a non-periodic axis needs Neumann on both sides (domain.cpp:85-129 leaves others unset)
    const char* ax[3][2] = {{"West", "East"}, {"South", "North"}, {"Front", "Back"}};
    for (auto& a : ax) {
        const std::string& lo = p.boundary_conditions.at(a[0]);
        const std::string& hi = p.boundary_conditions.at(a[1]);
        if (lo == "Periodic") continue;
        if (lo != "Neumann" || hi != "Neumann")
            return std::string("boundary pair ") + a[0] + "/" + a[1] + " = " + lo + "/" + hi +
                   " (a non-periodic axis needs Neumann on both sides)";
    }
    if (p.nx <= 0 || p.ny <= 0 || p.nz <= 0) return "grid sizes must be positive";
    return "";
}

ns_params to_ns_params(const Params& p, bool fp32) {
    ns_params q;
    ns_params_default(&q);
    q.dim = p.dim;
    q.nx = p.nx;
    q.ny = p.ny;
    q.nz = p.nz;
    q.Lx = p.Lx;
    q.Ly = p.Ly;
    q.Lz = p.Lz;
    q.mu = p.mu;
    q.Pr = p.Pr;
    q.gamma = p.gamma;
    q.cfl = p.CFL_max;
    // Driver::create_convection_operator (driver.cpp:74-92): CenteredConvection is
    // an empty operator in the reference, "none" the null one
    q.convection = p.convection_scheme != "Weno"
                       ? NS_CONV_NONE
                       : (p.convection_in_characteristic_space ? NS_CONV_WENO5_CHAR : NS_CONV_WENO5);
    q.weights = p.weight_type == "Borges" ? NS_WEIGHTS_BORGES : NS_WEIGHTS_SHU;
    // Driver::create_diffusion_operator (driver.cpp:94-105): only Centered acts
    q.diffusion = p.diffusion_scheme == "Centered" ? NS_DIFF_CENTERED : NS_DIFF_NONE;
    q.diffusion_order = p.diffusion_scheme_order;
    q.bc[0] = p.boundary_conditions.at("West") == "Periodic" ? NS_BC_PERIODIC : NS_BC_NEUMANN;
    q.bc[1] = p.boundary_conditions.at("South") == "Periodic" ? NS_BC_PERIODIC : NS_BC_NEUMANN;
    q.bc[2] = p.boundary_conditions.at("Front") == "Periodic" ? NS_BC_PERIODIC : NS_BC_NEUMANN;
    q.precision = fp32 ? NS_PREC_FP32 : NS_PREC_FP64;
    return q;
}

// ---------------------------------------------------------------------------
// initial conditions (src/testcases.cpp) on the host W array: AoS [i][j][k][q]
// with 3 ghost cells (q fastest), interior cells only, halos left at zero

struct HostField {
    int nx, ny, nz, NX, NY, NZ;
    std::vector<double> w;
    HostField(int x, int y, int z) : nx(x), ny(y), nz(z), NX(x + 6), NY(y + 6), NZ(z + 6) {
        w.assign((size_t)NX * NY * NZ * 5, 0.0);
    }
    double* at(int i, int j, int k) {  // interior indices
        return &w[((((size_t)(i + 3) * NY) + (j + 3)) * NZ + (k + 3)) * 5];
    }
};

// cell centre coordinate (Grid::create_point_coordinates, grid.cpp:34-54, one rank)
double centre(double L, int n, int i) {
    double d = L / n;
    return 0.0 + d * 0.5 + i * d;
}

typedef double State[5];

// set_quarters_xy / set_quarters_yz (testcases.cpp:140-260): "north-west" is
// a <= L_a/2 and y <= Ly/2, a = x or z
void quarters(HostField& F, const Params& p, bool yz, const State& NW, const State& NE, const State& SW,
              const State& SE) {
    for (int i = 0; i < F.nx; i++)
        for (int j = 0; j < F.ny; j++)
            for (int k = 0; k < F.nz; k++) {
                double a = yz ? centre(p.Lz, p.nz, k) : centre(p.Lx, p.nx, i);
                double La = yz ? p.Lz : p.Lx;
                double y = centre(p.Ly, p.ny, j);
                const double* s;
                if (a <= La / 2. && y <= p.Ly / 2.) s = NW;
                else if (a > La / 2. && y <= p.Ly / 2.) s = NE;
                else if (a <= La / 2. && y > p.Ly / 2.) s = SW;
                else s = SE;
                double* w = F.at(i, j, k);
                for (int q = 0; q < 5; q++) w[q] = s[q];
            }
}

// shear_layer_xy / shear_layer_3d (testcases.cpp:262-346): a stripe |y - Ly/2| <= width
// moving against the rest; the perturbations draw the C library's rand() in cell
// order, as the reference does (a fresh process starts its sequence the same way)
void shear(HostField& F, const Params& p, bool three_d) {
    const double pi = 3.14159265358979323846;
    const double stripe = (three_d ? 0.25 : 0.1) * p.Ly;
    for (int i = 0; i < F.nx; i++)
        for (int j = 0; j < F.ny; j++)
            for (int k = 0; k < F.nz; k++) {
                double x = centre(p.Lx, p.nx, i) - 0.5 * p.Lx;
                double y = centre(p.Ly, p.ny, j) - 0.5 * p.Ly;
                double* w = F.at(i, j, k);
                if (three_d) {
                    double zp = 0.02 * ((double)rand() / (RAND_MAX));
                    double yp = 0.02 * ((double)rand() / (RAND_MAX));
                    double vs = 0.01 * sin(2.0 * pi * x / p.Lx);
                    bool in = std::abs(y) <= stripe;
                    w[0] = in ? 2. : 1.;
                    w[1] = 2.5;
                    w[2] = in ? -0.5 : 0.5;
                    w[3] = in ? vs + yp : vs;
                    w[4] = zp;
                } else {
                    double yp = 0.01 * ((double)rand() / (RAND_MAX));
                    bool in = std::abs(y) <= stripe;
                    w[0] = 1.;
                    w[1] = 2.5;
                    w[2] = in ? -0.5 : 0.5;
                    w[3] = in ? yp : 0.0 * sin(2.0 * pi * x / p.Lx);
                    w[4] = 0.0;
                }
            }
}

bool set_initial_condition(HostField& F, const Params& p) {
    // left/right Sod states (testcases.cpp:5-58)
    const State L = {1., 1., 0., 0., 0.}, R = {0.125, 0.1, 0., 0., 0.};
    const std::string& c = p.testcase;
    if (c == "sod_x") quarters(F, p, false, L, R, L, R);
    else if (c == "sod_y") quarters(F, p, false, L, L, R, R);
    else if (c == "sod_z") quarters(F, p, true, L, R, L, R);
    // 2D Riemann problems (testcases.cpp:71-138)
    else if (c == "case3") {
        const State NW = {0.5323, 0.3, 1.206, 0., 0.}, NE = {1.5, 1.5, 0., 0., 0.},
                    SW = {0.138, 0.029, 1.206, -1.206, 0.}, SE = {0.5323, 0.3, 0., -1.206, 0.};
        quarters(F, p, false, NW, NE, SW, SE);
    } else if (c == "case4") {
        const State NW = {0.5065, 0.35, 0.8939, 0., 0.}, NE = {1.1, 1.1, 0., 0., 0.},
                    SW = {1.1, 1.1, 0.8939, -0.8938, 0.}, SE = {0.5065, 0.35, 0., -0.8939, 0.};
        quarters(F, p, false, NW, NE, SW, SE);
    } else if (c == "case6") {
        const State NW = {2.0, 1.0, 0.75, -0.5, 0.}, NE = {1.0, 1.0, 0.75, 0.5, 0.},
                    SW = {1.0, 1.0, -0.75, -0.5, 0.}, SE = {3.0, 1.0, -0.75, 0.5, 0.};
        quarters(F, p, false, NW, NE, SW, SE);
    } else if (c == "case12") {
        const State NW = {1.0, 1.0, 0.7276, 0., 0.}, NE = {0.5313, 0.4, 0., 0., 0.},
                    SW = {0.8, 1.0, 0., 0., 0.}, SE = {1.0, 1.0, 0., -0.7276, 0.};
        quarters(F, p, false, NW, NE, SW, SE);
    } else if (c == "case15") {
        const State NW = {0.5197, 0.4, -0.6259, 0.3, 0.}, NE = {1.0, 1.0, 0.1, 0.3, 0.},
                    SW = {0.8, 0.4, 0.1, 0.3, 0.}, SE = {0.5313, 0.4, 0.1, -0.4276, 0.};
        quarters(F, p, false, NW, NE, SW, SE);
    } else if (c == "case17") {
        // the reference's south-west state lists four values and reads a fifth past its
        // end (testcases.cpp:131); w = 0 here
        const State NW = {2.0, 1.0, 0., 0.3, 0.}, NE = {1.0, 1.0, 0., 0.4, 0.},
                    SW = {1.0625, 0.4, 0., -0.2145, 0.}, SE = {0.5197, 0.4, 0., 1.1259, 0.};
        quarters(F, p, false, NW, NE, SW, SE);
    } else if (c == "shear_xy") shear(F, p, false);
    else if (c == "shear_3d") shear(F, p, true);
    else return false;
    return true;
}

// ---------------------------------------------------------------------------
// output (BinaryWriter, io_binary.cpp) and checkpoints

bool make_dir(const std::string& d) {
    if (mkdir(d.c_str(), 0755) == 0 || errno == EEXIST) return true;
    return false;
}

bool write_fields(const std::string& dir, long long iter, double time, HostField& F) {
    std::string base = dir + "/fields_" + std::to_string(iter) + "_p_0";
    std::ofstream f(base + ".dat", std::ios::binary);
    if (!f) return false;
    for (int i = 0; i < F.nx; i++)
        for (int j = 0; j < F.ny; j++)
            for (int k = 0; k < F.nz; k++) f.write(reinterpret_cast<const char*>(F.at(i, j, k)), 5 * sizeof(double));
    if (!f) return false;
    std::ofstream t(base + ".time");
    t.precision(17);
    t << time << " " << iter << "\n";
    return (bool)t;
}

bool write_mesh(const std::string& dir, const Params& p) {
    std::ofstream f(dir + "/mesh_p_0.dat", std::ios::binary);
    if (!f) return false;
    for (int i = 0; i < p.nx; i++)
        for (int j = 0; j < p.ny; j++)
            for (int k = 0; k < p.nz; k++) {
                double c[3] = {centre(p.Lx, p.nx, i), centre(p.Ly, p.ny, j), centre(p.Lz, p.nz, k)};
                f.write(reinterpret_cast<const char*>(c), sizeof c);
            }
    return (bool)f;
}

bool read_checkpoint(const std::string& path, HostField& F, double& time, long long& iter, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path; return false; }
    for (int i = 0; i < F.nx; i++)
        for (int j = 0; j < F.ny; j++)
            for (int k = 0; k < F.nz; k++) f.read(reinterpret_cast<char*>(F.at(i, j, k)), 5 * sizeof(double));
    if (!f) { err = path + " holds fewer than nx*ny*nz*5 doubles"; return false; }
    if (f.peek() != EOF) { err = path + " holds more than nx*ny*nz*5 doubles"; return false; }
    std::string tpath = path;
    if (tpath.size() > 4 && tpath.compare(tpath.size() - 4, 4, ".dat") == 0) tpath.resize(tpath.size() - 4);
    std::ifstream t(tpath + ".time");
    if (!(t >> time >> iter)) { err = "cannot read time and iteration from " + tpath + ".time"; return false; }
    return true;
}

int usage() {
    std::cerr << "usage: ns_b200_driver [--input input.xml] [--precision fp64|fp32] [--results DIR]\n"
                 "                      [--max-steps N] [--restart FILE] [--check] [--dump-ic FILE]\n";
    return 2;
}

}  // namespace

int main(int argc, char** argv) {
    std::string input = "input.xml", results = "results", restart, dump_ic, precision = "fp64";
    long long max_steps = -1;
    bool check_only = false;
    for (int a = 1; a < argc; a++) {
        std::string k = argv[a];
        auto val = [&](std::string& v) {
            if (a + 1 >= argc) return false;
            v = argv[++a];
            return true;
        };
        std::string v;
        if (k == "--input") { if (!val(input)) return usage(); }
        else if (k == "--results") { if (!val(results)) return usage(); }
        else if (k == "--restart") { if (!val(restart)) return usage(); }
        else if (k == "--dump-ic") { if (!val(dump_ic)) return usage(); }
        else if (k == "--precision") { if (!val(precision) || (precision != "fp64" && precision != "fp32")) return usage(); }
        else if (k == "--max-steps") { if (!val(v)) return usage(); max_steps = atoll(v.c_str()); }
        else if (k == "--check") check_only = true;
        else return usage();
    }

    // Driver::read_parameters (driver.cpp:145-164)
    std::ifstream in(input);
    if (!in) {
        std::cerr << "File not found: " << input << std::endl;
        return 1;
    }
    std::stringstream ss;
    ss << in.rdbuf();
    std::string src = ss.str();
    XmlParser xp(src);
    XNode root;
    if (!xp.document(root)) {
        std::cerr << "Input file error: " << input << ": " << xp.err << std::endl;
        return 1;
    }
    Params p;
    try {
        p = read_input(root);
    } catch (const InputError& e) {
        std::cerr << "Input file error: missing or invalid " << e.what << std::endl;
        return 1;
    }
    std::string bad = sanity_check(p, !check_only);
    if (!bad.empty()) {
        std::cout << bad << std::endl;
        return 1;
    }
    bad = b200_limits(p);
    if (!bad.empty()) {
        std::cerr << "Not runnable: " << bad << std::endl;
        return 1;
    }
    const bool fp32 = precision == "fp32";
    ns_params q = to_ns_params(p, fp32);
    if (p.nproc_x * p.nproc_y * p.nproc_z != 1)
        std::cerr << "note: DomainDecomposition " << p.nproc_x << "x" << p.nproc_y << "x" << p.nproc_z
                  << " runs as one GPU domain" << std::endl;
    if (check_only) {
        std::cout.precision(17);
        std::cout << "{\"dim\": " << q.dim << ", \"nx\": " << q.nx << ", \"ny\": " << q.ny << ", \"nz\": " << q.nz
                  << ", \"Lx\": " << q.Lx << ", \"Ly\": " << q.Ly << ", \"Lz\": " << q.Lz << ", \"mu\": " << q.mu
                  << ", \"Pr\": " << q.Pr << ", \"gamma\": " << q.gamma << ", \"cfl\": " << q.cfl
                  << ", \"convection\": " << q.convection << ", \"weights\": " << q.weights
                  << ", \"diffusion\": " << q.diffusion << ", \"diffusion_order\": " << q.diffusion_order
                  << ", \"bc\": [" << q.bc[0] << ", " << q.bc[1] << ", " << q.bc[2] << "]"
                  << ", \"precision\": " << q.precision << ", \"end_t\": " << p.end_t
                  << ", \"io_interval\": " << p.io_interval << ", \"testcase\": \"" << p.testcase << "\""
                  << ", \"file_format\": \"" << p.output_file_format << "\"}" << std::endl;
        return 0;
    }

    HostField F(p.nx, p.ny, p.nz);
    double time = 0.0;
    long long iter = 0;
    if (!restart.empty()) {
        std::string err;
        if (!read_checkpoint(restart, F, time, iter, err)) {
            std::cerr << "Restart failed: " << err << std::endl;
            return 4;
        }
        std::cout << "Restarting from " << restart << " at time " << time << ", iteration " << iter << std::endl;
    } else if (!set_initial_condition(F, p)) {
        std::cerr << "Not runnable: test case " << p.testcase << std::endl;
        return 1;
    }
    if (!dump_ic.empty()) {
        std::ofstream f(dump_ic, std::ios::binary);
        f.write(reinterpret_cast<const char*>(F.w.data()), F.w.size() * sizeof(double));
        return f ? 0 : 4;
    }

    const bool write = p.io_interval > 0;
    if (p.output_file_format == "Hdf5")
        std::cerr << "note: this build has no HDF5; fields are written in the Binary layout" << std::endl;
    if (write && (!make_dir(results) || (restart.empty() && !write_mesh(results, p)))) {
        std::cerr << "cannot write to " << results << std::endl;
        return 4;
    }

    ns_ctx* ctx = nullptr;
    if (ns_create(&q, &ctx) != NS_OK) {
        std::cerr << "ns_create: " << ns_last_error_string() << std::endl;
        return 3;
    }
    auto lib_fail = [&](const char* what) {
        std::cerr << what << ": " << ns_last_error_string() << std::endl;
        ns_destroy(ctx);
        return 3;
    };
    if (ns_upload_primitive(ctx, F.w.data()) != NS_OK) return lib_fail("ns_upload_primitive");
    const double t0 = time;
    long long written = -1;
    auto dump = [&]() {
        if (ns_download_primitive(ctx, F.w.data()) != NS_OK) return 3;
        if (!write_fields(results, iter, time, F)) {
            std::cerr << "cannot write fields to " << results << std::endl;
            return 4;
        }
        written = iter;
        return 0;
    };

    // Driver::run's loop (driver.cpp:43-68)
    long long taken = 0;
    while (time < p.end_t && (max_steps < 0 || taken < max_steps)) {
        auto c0 = std::chrono::steady_clock::now();
        if (write && iter % p.io_interval == 0 && written != iter) {
            int rc = dump();
            if (rc) { ns_destroy(ctx); return rc; }
        }
        if (ns_advance(ctx, 1) != NS_OK) return lib_fail("ns_advance");
        double dt = 0.0, tsum = 0.0;
        if (ns_get_dt(ctx, &dt, &tsum) != NS_OK) return lib_fail("ns_get_dt");
        iter++;
        taken++;
        time = time + dt;
        double cpu = std::chrono::duration<double>(std::chrono::steady_clock::now() - c0).count();
        std::cout << "Flow time: " << time << "\tCPU time (step): " << cpu << "\tdt: " << dt
                  << "\tCFL: " << p.CFL_max << std::endl;
        if (!std::isfinite(dt)) break;
    }
    (void)t0;
    if (write && written != iter) {
        int rc = dump();
        if (rc) { ns_destroy(ctx); return rc; }
    }
    ns_diagnostics d;
    if (ns_get_diagnostics(ctx, &d) == NS_OK && d.nonfinite)
        std::cerr << "warning: the state holds NaN/Inf" << std::endl;
    ns_destroy(ctx);
    return 0;
}
