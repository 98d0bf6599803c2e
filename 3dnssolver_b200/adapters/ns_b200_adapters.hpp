// ns_b200_adapters.hpp -- the reference-side binding of the B200 path.
//
// Header-only C++ adapters that derive from the reference's own operator
// interfaces and forward to the C ABI of ns_b200.h.  A maintainer of the
// reference adds this header to its source tree (e.g. src/gpu/) and links
// libns_b200.so; compile it with the reference's include path.  It needs:
//   ConvectionScheme  (src/convection_schemes/convection_scheme.hpp:14-33)
//   DiffusionScheme   (src/diffusion_schemes/diffusion_scheme.hpp:11-19)
//   Domain, Grid, Communicator, Params (src/domain.hpp, src/grid.hpp,
//   src/communicator.hpp, src/params.hpp)
// Scope: one rank (the context's box is the whole periodic/Neumann domain).
#ifndef NS_B200_ADAPTERS_HPP
#define NS_B200_ADAPTERS_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "ns_b200.h"

namespace ns_b200 {

// Params (src/params.hpp:20-43) -> ns_params for a single-rank run
inline ns_params to_ns_params(const Params& p) {
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
    q.convection = p.convection_scheme != "Weno"
                       ? NS_CONV_NONE
                       : (p.convection_in_characteristic_space ? NS_CONV_WENO5_CHAR : NS_CONV_WENO5);
    q.weights = p.weight_type == "Borges" ? NS_WEIGHTS_BORGES : NS_WEIGHTS_SHU;
    q.diffusion = p.diffusion_scheme == "Centered" ? NS_DIFF_CENTERED : NS_DIFF_NONE;
    q.diffusion_order = p.diffusion_scheme_order;
    // periodicity follows West/South/Front like Decomposition (src/decomposition.cpp:145-161)
    auto bc = [&](const char* side) {
        return p.boundary_conditions.at(side) == "Periodic" ? NS_BC_PERIODIC : NS_BC_NEUMANN;
    };
    q.bc[0] = bc("West");
    q.bc[1] = bc("South");
    q.bc[2] = bc("Front");
    return q;
}

// Address of an Array4d's storage.  The reference's const accessor returns by
// value (src/containers/array_4d.hpp:64-67) and the class has no data(), so the
// non-const accessor gives the address; the B200 calls only read inputs.
inline const double* data(const Array4d& a) { return &const_cast<Array4d&>(a)(0, 0, 0, 0); }
inline double* data(Array4d& a) { return &a(0, 0, 0, 0); }

inline void check(ns_status s, const char* what) {
    if (s != NS_OK) throw std::runtime_error(std::string(what) + ": " + ns_last_error_string());
}

// One device context for the run (owns the device state and stream).
class Context {
public:
    explicit Context(const Params& p) {
        ns_params q = to_ns_params(p);
        check(ns_create(&q, &m_ctx), "ns_create");
        m_elems = ns_host_array_elems(&q);
    }
    ~Context() { ns_destroy(m_ctx); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    ns_ctx* get() const { return m_ctx; }
    size_t host_elems() const { return m_elems; }  // doubles of one host Array4d

private:
    ns_ctx* m_ctx = nullptr;
    size_t m_elems = 0;
};

// ConvectionScheme::solve(grid, W, U, R): R += convective residual on the GPU
class GpuConvection : public ConvectionScheme {
public:
    GpuConvection(Context& c, double gamma) : ConvectionScheme("Weno-5 B200", gamma), m_c(c) {}
    void solve(const Grid&, const Array4d& W, const Array4d& U, Array4d& R) override {
        check(ns_convection_solve(m_c.get(), data(W), data(U), data(R)), "ns_convection_solve");
    }

private:
    Context& m_c;
};

// DiffusionScheme::solve(grid, comm, W, R): R += viscous residual on the GPU
class GpuDiffusion : public DiffusionScheme {
public:
    GpuDiffusion(Context& c, const Params& p)
        : DiffusionScheme("Centered B200", p.gamma, p.mu, p.Pr), m_c(c) {}
    void solve(const Grid&, const Communicator&, const Array4d& W, Array4d& R) override {
        check(ns_diffusion_solve(m_c.get(), data(W), data(R)), "ns_diffusion_solve");
    }

private:
    Context& m_c;
};

// TimeScheme::step (src/time_scheme.hpp:25-29) with the whole step on the GPU:
// W is uploaded, stepped and downloaded with U each call.
// With pin (the default) the first step page-locks the Domain's W and U
// (ns_host_register), so that every step overlaps its copies with the stages;
// the destructor releases them, so destroy the scheme before the Domain.  A
// range that cannot be locked is used as it is.
class GpuTimeScheme {
public:
    explicit GpuTimeScheme(Context& c, bool pin = true) : m_c(c), m_pin(pin) {}
    ~GpuTimeScheme() {
        for (double* p : m_pinned) ns_host_unregister(p);
    }
    GpuTimeScheme(const GpuTimeScheme&) = delete;
    GpuTimeScheme& operator=(const GpuTimeScheme&) = delete;
    void step(Domain& d, const Grid&, const Communicator&, ConvectionScheme*, DiffusionScheme*) {
        double* W = data(d.get_NS_primitive_array());
        double* U = data(d.get_NS_conservative_array());
        if (m_pin) {
            m_pin = false;
            for (double* p : {W, U})
                if (ns_host_register(p, m_c.host_elems() * sizeof(double)) == NS_OK) m_pinned.push_back(p);
        }
        check(ns_time_step(m_c.get(), W, U, &m_dt), "ns_time_step");
    }
    double get_dt() const { return m_dt; }

private:
    Context& m_c;
    bool m_pin;
    std::vector<double*> m_pinned;
    double m_dt = 0.0;
};

}  // namespace ns_b200

#endif
