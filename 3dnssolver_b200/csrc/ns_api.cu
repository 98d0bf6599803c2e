// ns_api.cu -- the C ABI of include/ns_b200.h: context, validation, host
// transfers and the orchestration of the RK3 stage kernels on one stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <utility>
#include <new>
#include <string>
#include <vector>

#include "ns_common.cuh"
#include "ns_kernels.h"
#include "ns_sensor.h"

using namespace nsb;

namespace {

thread_local std::string g_err;

ns_status fail(ns_status s, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
ns_status fail(ns_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return s;
}

#define NS_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(e_ == cudaErrorMemoryAllocation ? NS_ERR_OOM : NS_ERR_CUDA, "%s: %s", \
                        #call, cudaGetErrorString(e_));                                     \
    } while (0)

#define NS_TRY(expr)                 \
    do {                             \
        ns_status s_ = (expr);       \
        if (s_ != NS_OK) return s_;  \
    } while (0)

}  // namespace

struct ns_ctx {
    ns_params p;
    Box box;
    FaceBox fb[3];
    Consts c;
    int device = 0;
    cudaStream_t own = nullptr, stream = nullptr;
    double* W = nullptr;   // primitive, halo'd SoA
    double* U = nullptr;   // conservative, halo'd SoA
    double* U0 = nullptr;  // RK stage base (interior used)
    double* U2 = nullptr;  // second stage buffer of the fused paths
    bool xfused = false;   // FP64 steps: x-faces and update in one kernel (k_xface_update)
    double* W2 = nullptr;  // its second W buffer (the next stage's W)
    bool w_next_ready = false;  // with fused_ready: W holds prim(U0) for the next step's first stage
    double* R = nullptr;   // residual for the operator entry points (lazy)
    void* F[3] = {nullptr, nullptr, nullptr};
    double* stage = nullptr;              // host-layout staging (lazy)
    unsigned long long* slot = nullptr;   // [0],[1]: CFL minima by step parity, [2]: scratch
    double* diag = nullptr;               // [8] diagnostics sums
    double* clock = nullptr;              // [2] last dt, accumulated time
    bool w_valid = false, u_valid = false;
    bool fused = false;        // steps run as one fused kernel per stage
    bool fused_ready = false;  // U0 holds the next step's start and slot[parity] its CFL minimum
    bool halos_stale = false;  // U's ghost cells predate the last fused step
    int parity = 0;
    long long steps = 0;
    long long launches = 0;
    nsb::SensorState* sensor = nullptr;
    double last_sensor_fraction = 0.0;
    // slab decomposition: the exchange callback and, while it runs, what it exchanges
    ns_exchange_fn xfn = nullptr;
    void* xuser = nullptr;
    int xwhat = -1;
    double* xbuf = nullptr;                  // the stage input whose ghost planes are exchanged
    unsigned long long* xslot = nullptr;     // the CFL minimum reduced over the slabs
    bool flags_valid = false;                // the sensor's flags belong to the current state's run
    int sms = 148;                           // multiprocessors of the context's device
    nsb::WTmaMaps tma[2];                    // FP64 steps: tensor maps of W and W2 (face tiles, viscous planes)
    // ns_time_step's transfer pipeline: the copy stream and its events (lazy)
    cudaStream_t copy = nullptr;
    std::vector<cudaEvent_t> ev;
};

static size_t host_elems(const ns_params* p) {
    return (size_t)(p->nx + 2 * NS_NGC) * (p->ny + 2 * NS_NGC) * (p->nz + 2 * NS_NGC) * NS_NQ;
}

static ns_status validate(const ns_params* p) {
    if (!p) return fail(NS_ERR_INVALID_ARG, "params is NULL");
    if (p->dim != 2 && p->dim != 3) return fail(NS_ERR_INVALID_ARG, "dim must be 2 or 3 (got %d)", p->dim);
    if (p->nx < 3 || p->ny < 3 || p->nz < 1 || (p->dim == 3 && p->nz < 3))
        return fail(NS_ERR_INVALID_ARG,
                    "grid %dx%dx%d: need nx, ny >= 3 and nz >= 3 when dim == 3 (3 ghost cells per side)",
                    p->nx, p->ny, p->nz);
    if ((long long)p->nx + 6 > 65535)
        return fail(NS_ERR_INVALID_ARG, "nx = %d exceeds the launch grid limit", p->nx);
    if (!(p->Lx > 0 && p->Ly > 0 && p->Lz > 0)) return fail(NS_ERR_INVALID_ARG, "domain lengths must be > 0");
    if (!(p->gamma > 1.0)) return fail(NS_ERR_INVALID_ARG, "gamma must be > 1");
    if (!(p->mu >= 0.0)) return fail(NS_ERR_INVALID_ARG, "mu must be >= 0");
    if (!(p->Pr > 0.0)) return fail(NS_ERR_INVALID_ARG, "Pr must be > 0");
    if (!(p->cfl > 0.0)) return fail(NS_ERR_INVALID_ARG, "cfl must be > 0");
    if (p->convection < NS_CONV_NONE || p->convection > NS_CONV_WENO5_CHAR)
        return fail(NS_ERR_INVALID_ARG, "unknown convection scheme %d", p->convection);
    if (p->weights != NS_WEIGHTS_SHU && p->weights != NS_WEIGHTS_BORGES)
        return fail(NS_ERR_INVALID_ARG, "unknown WENO weight type %d", p->weights);
    if (p->diffusion != NS_DIFF_NONE && p->diffusion != NS_DIFF_CENTERED)
        return fail(NS_ERR_INVALID_ARG, "unknown diffusion scheme %d", p->diffusion);
    if (p->diffusion_order != 2 && p->diffusion_order != 4 && p->diffusion_order != 6)
        return fail(NS_ERR_INVALID_ARG, "diffusion order must be 2, 4 or 6 (got %d)", p->diffusion_order);
    for (int a = 0; a < 3; a++)
        if (p->bc[a] != NS_BC_PERIODIC && p->bc[a] != NS_BC_NEUMANN && !(a == 0 && p->bc[a] == NS_BC_EXTERNAL))
            return fail(NS_ERR_INVALID_ARG, "unknown boundary type %d on axis %d%s", p->bc[a], a,
                        p->bc[a] == NS_BC_EXTERNAL ? " (NS_BC_EXTERNAL is for the x axis only)" : "");
    if (p->bc[0] == NS_BC_EXTERNAL) {
        if (p->slab_nx < p->nx || p->slab_x0 < 0 || (long long)p->slab_x0 + p->nx > p->slab_nx)
            return fail(NS_ERR_INVALID_ARG, "slab x0 = %d, nx = %d does not lie inside a domain of %d cells",
                        p->slab_x0, p->nx, p->slab_nx);
        if (p->slab_periodic != 0 && p->slab_periodic != 1)
            return fail(NS_ERR_INVALID_ARG, "slab_periodic must be 0 or 1");
        if (p->sensor) return fail(NS_ERR_INVALID_ARG, "the sensor-gated form runs on a single domain");
    }
    if (p->precision != NS_PREC_FP64 && p->precision != NS_PREC_FP32)
        return fail(NS_ERR_INVALID_ARG, "unknown precision %d", p->precision);
    if (p->semantics != NS_SEM_REFERENCE && p->semantics != NS_SEM_PHYSICAL)
        return fail(NS_ERR_INVALID_ARG, "unknown semantics %d", p->semantics);
    if (p->check_finite != 0 && p->check_finite != 1)
        return fail(NS_ERR_INVALID_ARG, "check_finite must be 0 or 1 (got %d)", p->check_finite);
    if (p->sensor) {
        if (p->convection != NS_CONV_WENO5_CHAR)
            return fail(NS_ERR_INVALID_ARG, "the sensor gates the characteristic scheme: convection must be NS_CONV_WENO5_CHAR");
        if (p->precision != NS_PREC_FP32)
            return fail(NS_ERR_INVALID_ARG, "the sensor-gated form runs in NS_PREC_FP32");
        if (!(p->sensor_threshold > 0.0 && p->sensor_threshold < 1.0))
            return fail(NS_ERR_INVALID_ARG, "sensor_threshold must lie in (0,1)");
        if (p->sensor_period < 0) return fail(NS_ERR_INVALID_ARG, "sensor_period must be >= 0");
    }
    return NS_OK;
}

static Consts make_consts(const ns_params* p) {
    // CD coefficients, src/difference_operators/cd_constants.hpp:10-28 (centred at index 3)
    static const double cd2_df[3] = {-1. / 2, 0., 1. / 2.};
    static const double cd2_ddf[3] = {1., -2., 1.};
    static const double cd4_df[5] = {1. / 12., -2. / 3., 0., 2. / 3., -1. / 12.};
    static const double cd4_ddf[5] = {-1. / 12., 4. / 3., -5. / 2., 4. / 3., -1. / 12.};
    static const double cd6_df[7] = {-1. / 60., 3. / 20., -3. / 4., 0., 3. / 4., -3. / 20., 1. / 60.};
    static const double cd6_ddf[7] = {1. / 90., -3. / 20., 3. / 2., -49. / 18., 3. / 2., -3. / 20., 1. / 90.};
    Consts c;
    memset(&c, 0, sizeof c);
    c.gamma = p->gamma;
    c.gm1 = p->gamma - 1.0;
    c.inv_gm1 = 1.0 / (p->gamma - 1.0);
    c.mu = p->mu;
    c.lamb = (-2. / 3.) * p->mu;
    c.heat = p->gamma / (p->Pr * (p->gamma - 1.0));
    c.dx = p->Lx / p->nx;
    c.dy = p->Ly / p->ny;
    c.dz = p->Lz / p->nz;
    c.inv_dx = 1.0 / c.dx;
    c.inv_dy = 1.0 / c.dy;
    c.inv_dz = 1.0 / c.dz;
    c.cfl = p->cfl;
    for (int a = 0; a < 3; a++) c.periodic[a] = (p->bc[a] == NS_BC_PERIODIC);
    c.ext_x = p->bc[0] == NS_BC_EXTERNAL;
    c.x0 = c.ext_x ? p->slab_x0 : 0;
    c.nxg = c.ext_x ? p->slab_nx : p->nx;
    c.xper = c.ext_x ? p->slab_periodic : c.periodic[0];
    c.dim = p->dim;
    c.order = p->diffusion_order;
    const double *df = cd2_df, *ddf = cd2_ddf;
    int w = 3;
    if (p->diffusion_order == 4) { df = cd4_df; ddf = cd4_ddf; w = 5; }
    if (p->diffusion_order == 6) { df = cd6_df; ddf = cd6_ddf; w = 7; }
    int h = w / 2;
    for (int t = 0; t < w; t++) {
        c.df[3 - h + t] = df[t];
        c.ddf[3 - h + t] = ddf[t];
    }
    return c;
}

static size_t soa_bytes(const Box& b) { return (size_t)b.fstride * NS_NQ * sizeof(double); }

static ns_status check_launch(ns_ctx* ctx, int n) {
    ctx->launches += n;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NS_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    return NS_OK;
}

static ns_status ensure_stage(ns_ctx* ctx) {
    if (!ctx->stage) NS_CUDA(cudaMalloc(&ctx->stage, host_elems(&ctx->p) * sizeof(double)));
    return NS_OK;
}

static ns_status ensure_R(ns_ctx* ctx) {
    if (!ctx->R) {
        NS_CUDA(cudaMalloc(&ctx->R, soa_bytes(ctx->box)));
        NS_CUDA(cudaMemsetAsync(ctx->R, 0, soa_bytes(ctx->box), ctx->stream));
    }
    return NS_OK;
}

static ns_status upload(ns_ctx* ctx, const double* host, double* dev) {
    if (!host) return fail(NS_ERR_INVALID_ARG, "host array is NULL");
    NS_TRY(ensure_stage(ctx));
    NS_CUDA(cudaMemcpyAsync(ctx->stage, host, host_elems(&ctx->p) * sizeof(double),
                            cudaMemcpyHostToDevice, ctx->stream));
    launch_aos_to_soa(ctx->stage, dev, ctx->box, ctx->stream);
    return check_launch(ctx, 1);
}

static ns_status download(ns_ctx* ctx, const double* dev, double* host) {
    if (!host) return fail(NS_ERR_INVALID_ARG, "host array is NULL");
    NS_TRY(ensure_stage(ctx));
    launch_soa_to_aos(dev, ctx->stage, ctx->box, ctx->stream);
    NS_TRY(check_launch(ctx, 1));
    NS_CUDA(cudaMemcpyAsync(host, ctx->stage, host_elems(&ctx->p) * sizeof(double),
                            cudaMemcpyDeviceToHost, ctx->stream));
    NS_CUDA(cudaStreamSynchronize(ctx->stream));
    return NS_OK;
}

static bool phys(const ns_ctx* ctx) { return ctx->p.semantics == NS_SEM_PHYSICAL; }
static bool slab(const ns_ctx* ctx) { return ctx->p.bc[0] == NS_BC_EXTERNAL; }

// Slab decomposition: hands the step to the exchange callback (halo planes of the
// stage input `buf`, or the CFL minimum `slot`); nothing to do on a single domain.
static ns_status exchange(ns_ctx* ctx, int what, double* buf, unsigned long long* slot) {
    if (!slab(ctx)) return NS_OK;
    if (!ctx->xfn) return fail(NS_ERR_INVALID_ARG, "a slab context (bc[0] = NS_BC_EXTERNAL) steps only with an "
                                                   "exchange callback (ns_set_exchange)");
    ctx->xwhat = what;
    ctx->xbuf = buf;
    ctx->xslot = slot;
    g_err.clear();
    ns_status st = ctx->xfn(ctx->xuser, ctx, what, (void*)ctx->stream);
    ctx->xwhat = -1;
    ctx->xbuf = nullptr;
    ctx->xslot = nullptr;
    if (st != NS_OK && g_err.empty()) return fail(st, "the exchange callback failed (%s)", what ? "halo" : "dt");
    return st;
}
static bool fp32(const ns_ctx* ctx) { return ctx->p.precision == NS_PREC_FP32; }

// optional event trail for ns_profile_step: an event after every kernel, tagged
// with the kernel class it closes
struct Prof {
    cudaEvent_t ev[64];
    int cls[64];
    int n = 0;
};
static Prof* g_prof = nullptr;  // set only inside ns_profile_step (single-threaded per context)

static void prof_mark(ns_ctx* ctx, int cls) {
    if (!g_prof || g_prof->n >= 64) return;
    cudaEventRecord(g_prof->ev[g_prof->n], ctx->stream);
    g_prof->cls[g_prof->n++] = cls;
}

// TMA-staged FP64 kernels: the y/z faces and the viscous terms of the physical
// semantics, the x-march of both (build switches, on by default)
#ifndef NS_FACE_TMA
#define NS_FACE_TMA 1
#endif
#ifndef NS_VISC_TMA_MAX_ORDER
#define NS_VISC_TMA_MAX_ORDER 6  // CD orders whose viscous terms march over TMA planes
#endif
#ifndef NS_VISC_TMA_REF
#define NS_VISC_TMA_REF 1  // the reference semantics' viscous terms too
#endif
#ifndef NS_XUPD_TMA
#define NS_XUPD_TMA 1
#endif
#ifndef NS_FACE_TMA_REF
#define NS_FACE_TMA_REF 0  // the TMA face tiles for the reference semantics' y/z faces too
#endif

// the TMA tensor maps of the context's current W (FP64 steps), or null
static const nsb::WTmaMaps* tma_maps(const ns_ctx* ctx) {
    if (fp32(ctx)) return nullptr;
    for (const nsb::WTmaMaps& t : ctx->tma)
        if (t.ok && t.W == ctx->W) return &t;
    return nullptr;
}

// face fluxes of the current (W, U) along every convected axis from first_dir on
// (U: the context's, or the stage input Uin); pl: the x-planes of the y- and
// z-faces of an FP64 time step (w_only), all planes by default
static ns_status faces(ns_ctx* ctx, int first_dir = 0, const double* Uin = nullptr, bool w_only = false,
                       Planes pl = Planes()) {
    const ns_params& p = ctx->p;
    const double* U = Uin ? Uin : ctx->U;
    if (p.convection == NS_CONV_NONE) return NS_OK;
    int nd = p.dim == 3 ? 3 : 2;
    for (int d = first_dir; d < nd; d++) {
        if (p.sensor) {
            if (sensor_face_flux(ctx->sensor, d, ctx->W, ctx->U, ctx->box, ctx->c, p.sensor_threshold,
                                 p.weights == NS_WEIGHTS_BORGES, phys(ctx), ctx->F[d], ctx->fb[d], ctx->stream,
                                 &ctx->launches) != NS_OK)
                return fail(NS_ERR_CUDA, "gated face kernel launch failed: %s",
                            cudaGetErrorString(cudaGetLastError()));
        } else {
            // the TMA tiles serve the physical semantics, whose face stencils read
            // every cell twice (local LF speed, then the split): from shared memory
            // that is 7-8% faster than the per-thread kernels on B200, which are 3-7%
            // faster for the reference semantics' single pass (256^3)
            const nsb::WTmaMaps* m =
                (NS_FACE_TMA && w_only && d > 0 && (phys(ctx) || NS_FACE_TMA_REF)) ? tma_maps(ctx) : nullptr;
            if (m)
                launch_face_flux_tma(d, p.convection == NS_CONV_WENO5_CHAR, p.weights == NS_WEIGHTS_BORGES,
                                     phys(ctx), *m, ctx->W, ctx->box, ctx->c, ctx->F[d], ctx->fb[d], ctx->sms,
                                     ctx->slot + 4, ctx->stream, pl);
            else
                launch_face_flux(d, p.convection == NS_CONV_WENO5_CHAR, p.weights == NS_WEIGHTS_BORGES,
                                 phys(ctx), fp32(ctx), ctx->W, U, ctx->box, ctx->c, ctx->F[d],
                                 ctx->fb[d], ctx->stream, w_only, w_only ? pl : Planes());
            NS_TRY(check_launch(ctx, d > 0 ? 2 : 1));  // y and z: the face grid and its last plane
        }
        prof_mark(ctx, NS_PROF_FACE_X + d);
    }
    return NS_OK;
}

static UpdateArgs update_args(ns_ctx* ctx, int mode, bool conv, bool visc) {
    UpdateArgs a;
    memset(&a, 0, sizeof a);
    a.W = ctx->W;
    a.U = ctx->U;
    a.U0 = ctx->U0;
    for (int d = 0; d < 3; d++) { a.F[d] = ctx->F[d]; a.fb[d] = ctx->fb[d]; }
    a.b = ctx->box;
    a.c = ctx->c;
    a.flags = 0;
    if (conv && ctx->p.convection != NS_CONV_NONE) {
        a.flags |= UPD_CONV;
        if (ctx->p.dim == 3) a.flags |= UPD_CONVZ;
    }
    a.mode = mode;
    a.viscous = visc && ctx->p.diffusion == NS_DIFF_CENTERED;
    a.phys = phys(ctx);
    a.fp32 = fp32(ctx);
    a.slot = ctx->slot;
    a.Rout = ctx->R;
    return a;
}

// one TimeScheme::step as one fused kernel per stage
static ns_status do_step_fused(ns_ctx* ctx) {
    cudaStream_t s = ctx->stream;
    unsigned long long* cur = ctx->slot + ctx->parity;
    unsigned long long* nxt = ctx->slot + (ctx->parity ^ 1);
    if (!ctx->fused_ready) {
        // dt from W at the step start (set_dt) and U0 = cons(W) (time_scheme.cpp:124-126)
        NS_CUDA(cudaMemsetAsync(cur, 0xFF, sizeof(unsigned long long), s));
        launch_step_begin(!ctx->w_valid, phys(ctx), ctx->W, ctx->U, ctx->U0, ctx->box, ctx->c, cur, s);
        NS_TRY(check_launch(ctx, 1));
        prof_mark(ctx, NS_PROF_STEP_BEGIN);
    }
    NS_CUDA(cudaMemsetAsync(nxt, 0xFF, sizeof(unsigned long long), s));
    const ns_params& p = ctx->p;
    FusedArgs a;
    memset(&a, 0, sizeof a);
    a.b = ctx->box;
    a.c = ctx->c;
    a.conv_dims = p.convection == NS_CONV_NONE ? 0 : (p.dim == 3 ? 3 : 2);
    a.visc_h = p.diffusion == NS_DIFF_CENTERED ? p.diffusion_order / 2 : 0;
    a.fp32 = fp32(ctx);
    a.chr = p.convection == NS_CONV_WENO5_CHAR;
    a.borges = p.weights == NS_WEIGHTS_BORGES;
    a.phys = phys(ctx);
    a.U0 = ctx->U0;
    a.slot = cur;
    a.slot_next = nxt;
    const bool gated = p.sensor && a.conv_dims > 0;
    GateLists gl;
    if (gated) {
        // the network on the step's start state (every sensor_period steps); its
        // flags gate the three stages: component-wise stages, then the flagged
        // faces corrected to characteristic-wise (ns_gate.cu)
        const int period = p.sensor_period > 1 ? p.sensor_period : 1;
        if (!ctx->flags_valid || ctx->steps % period == 0) {
            if (sensor_step_flags(ctx->sensor, ctx->U0, ctx->box, ctx->c, p.sensor_threshold, ctx->fb, a.conv_dims, s,
                                  &ctx->launches) != NS_OK)
                return fail(NS_ERR_CUDA, "sensor flag kernels failed: %s", cudaGetErrorString(cudaGetLastError()));
            ctx->flags_valid = true;
            prof_mark(ctx, NS_PROF_SENSOR);
        }
        gl = sensor_gate_lists(ctx->sensor);
        a.chr = false;
        a.skip = gl.touched;
    }
    // SSP-RK3 coefficients (time_scheme.cpp:36-38, 48-50, 60-62); U0 -> U -> U2 -> U
    const double m1[3] = {1.0, 3.0 / 4.0, 1. / 3.};
    const double m2[3] = {0.0, 1.0 / 4.0, 2. / 3.};
    const double mc[3] = {-1.0, -(1. / 4.), -(2. / 3.)};
    double* in[3] = {ctx->U0, ctx->U, ctx->U2};
    double* out[3] = {ctx->U, ctx->U2, ctx->U};
    NS_TRY(exchange(ctx, NS_EXCHANGE_DT, nullptr, cur));
    for (int st = 0; st < 3; st++) {
        NS_TRY(exchange(ctx, NS_EXCHANGE_HALO, in[st], nullptr));
        a.Uin = in[st];
        a.Uout = out[st];
        a.m1 = m1[st];
        a.m2 = m2[st];
        a.mc = mc[st];
        a.last = (st == 2);
        a.clock = (st == 0) ? ctx->clock : nullptr;
        cudaError_t e = launch_stage_fused(a, s);
        ctx->launches++;
        if (e != cudaSuccess) return fail(NS_ERR_CUDA, "fused stage launch failed: %s", cudaGetErrorString(e));
        prof_mark(ctx, NS_PROF_STAGE_FUSED);
        if (gated) {
            e = gate_correct(a, gl, ctx->F, ctx->fb, ctx->sms, s);
            ctx->launches += a.conv_dims + 1;
            if (e != cudaSuccess) return fail(NS_ERR_CUDA, "sensor correction launch failed: %s", cudaGetErrorString(e));
            prof_mark(ctx, NS_PROF_SENSOR);
        }
    }
    ctx->parity ^= 1;
    ctx->fused_ready = true;
    ctx->halos_stale = true;
    ctx->u_valid = true;
    ctx->w_valid = false;
    ctx->steps++;
    return NS_OK;
}

// SSP-RK3 coefficients (time_scheme.cpp:36-38, 48-50, 60-62): U = U0 m1 + U m2 + R (mc dt)
static const double kRkM1[3] = {1.0, 3.0 / 4.0, 1. / 3.};
static const double kRkM2[3] = {0.0, 1.0 / 4.0, 2. / 3.};
static const double kRkMc[3] = {-1.0, -(1. / 4.), -(2. / 3.)};

// FP64 stage st after its fill, on the x-planes pl: the y- and z-faces (with
// faces), the viscous terms, then the x-faces marched together with the cell
// update from Uin into Uout (and the next stage's W into W2)
static ns_status xstage(ns_ctx* ctx, int st, double* Uin, double* Uout, unsigned long long* cur,
                        unsigned long long* nxt, bool with_faces, Planes pl) {
    cudaStream_t s = ctx->stream;
    if (with_faces) NS_TRY(faces(ctx, 1, Uin, true, pl));  // W = prim(U) here: the stencils read W only
    UpdateArgs a = update_args(ctx, MODE_STAGE, true, true);
    if (a.viscous) {  // into the x-face array, which the x-march leaves unused
        a.V = (const double*)ctx->F[0];
        a.vs = ctx->fb[0].fstride;
        const nsb::WTmaMaps* m = tma_maps(ctx);
        if (m && ctx->c.order <= NS_VISC_TMA_MAX_ORDER && (phys(ctx) || NS_VISC_TMA_REF))
            launch_viscous_tma(ctx->c.order / 2, phys(ctx), *m, ctx->W, ctx->box, ctx->c, (double*)ctx->F[0],
                               ctx->fb[0].fstride, ctx->slot + 4, s, pl);
        else if (pl.n < 0)
            launch_viscous(ctx->c.order / 2, phys(ctx), ctx->W, ctx->box, ctx->c, (double*)ctx->F[0],
                           ctx->fb[0].fstride, s);
        else
            return fail(NS_ERR_UNSUPPORTED, "a plane range of the viscous terms needs their TMA kernel");
        NS_TRY(check_launch(ctx, 1));
        prof_mark(ctx, NS_PROF_VISCOUS);
    }
    a.U = Uin;
    a.Unext = Uout;
    a.Wnext = ctx->W2;
    a.slot = cur;
    a.slot_next = (st == 2) ? nxt : nullptr;
    a.m1 = kRkM1[st];
    a.m2 = kRkM2[st];
    a.mc = kRkMc[st];
    a.clock = (st == 0) ? ctx->clock : nullptr;
    const nsb::WTmaMaps* xm = NS_XUPD_TMA ? tma_maps(ctx) : nullptr;
    if (xm)
        launch_xface_update_tma(ctx->p.convection == NS_CONV_WENO5_CHAR, ctx->p.weights == NS_WEIGHTS_BORGES, a, *xm,
                                ctx->slot + 4, s, pl);
    else if (pl.n < 0)
        launch_xface_update(ctx->p.convection == NS_CONV_WENO5_CHAR, ctx->p.weights == NS_WEIGHTS_BORGES, a, s);
    else
        return fail(NS_ERR_UNSUPPORTED, "a plane range of the x-march needs its TMA kernel");
    NS_TRY(check_launch(ctx, 1));
    prof_mark(ctx, NS_PROF_XFACE_UPDATE);
    return NS_OK;
}

// the state after an FP64 step of do_step: U holds it, U0 and the other parity
// slot the next step's start, W (after the last swap) the next stage's W
static void end_xstep(ns_ctx* ctx) {
    ctx->parity ^= 1;
    ctx->fused_ready = true;
    ctx->w_next_ready = true;
    ctx->u_valid = true;
    ctx->w_valid = false;
    ctx->steps++;
}

// one TimeScheme::step on the device state
static ns_status do_step(ns_ctx* ctx) {
    if (ctx->fused) return do_step_fused(ctx);
    cudaStream_t s = ctx->stream;
    unsigned long long* cur = ctx->slot + ctx->parity;
    if (!ctx->xfused) {
        NS_CUDA(cudaMemsetAsync(cur, 0xFF, sizeof(unsigned long long), s));
        launch_step_begin(!ctx->w_valid, phys(ctx), ctx->W, ctx->U, ctx->U0, ctx->box, ctx->c, cur, s);
        NS_TRY(check_launch(ctx, 1));
        prof_mark(ctx, NS_PROF_STEP_BEGIN);
        NS_TRY(exchange(ctx, NS_EXCHANGE_DT, nullptr, cur));
        for (int st = 0; st < 3; st++) {
            NS_TRY(exchange(ctx, NS_EXCHANGE_HALO, ctx->U, nullptr));
            launch_fill_prim(ctx->W, ctx->U, ctx->box, ctx->c, s);
            NS_TRY(check_launch(ctx, 1));
            prof_mark(ctx, NS_PROF_FILL);
            NS_TRY(faces(ctx));
            UpdateArgs a = update_args(ctx, MODE_STAGE, true, true);
            a.slot = cur;
            a.m1 = kRkM1[st];
            a.m2 = kRkM2[st];
            a.mc = kRkMc[st];
            a.clock = (st == 0) ? ctx->clock : nullptr;
            launch_update(a, s);
            NS_TRY(check_launch(ctx, 1));
            prof_mark(ctx, NS_PROF_UPDATE);
        }
        ctx->u_valid = true;
        ctx->w_valid = false;
        ctx->steps++;
        return NS_OK;
    }
    // FP64 with convection: per stage the fill, the y- and z-faces, then the
    // x-faces marched together with the cell update into the other buffer:
    // U0 -> U -> U2 -> U (stage 1 reads the step's start U0 directly).  The
    // fill copies the stage input's halos into the output buffer, so the step
    // ends with the halos the reference's U holds.  The third stage also forms
    // the next step's start (U0, and the CFL minimum in the other parity slot),
    // so only the first step after a state change runs k_step_begin.
    unsigned long long* nxt = ctx->slot + (ctx->parity ^ 1);
    if (!ctx->fused_ready) {
        NS_CUDA(cudaMemsetAsync(cur, 0xFF, sizeof(unsigned long long), s));
        launch_step_begin(!ctx->w_valid, phys(ctx), ctx->W, ctx->U, ctx->U0, ctx->box, ctx->c, cur, s);
        NS_TRY(check_launch(ctx, 1));
        prof_mark(ctx, NS_PROF_STEP_BEGIN);
    }
    NS_CUDA(cudaMemsetAsync(nxt, 0xFF, sizeof(unsigned long long), s));
    double* in[3] = {ctx->U0, ctx->U, ctx->U2};
    double* out[3] = {ctx->U, ctx->U2, ctx->U};
    // W's interior for a stage is the previous x-update's output (W and W2 swap
    // each stage); the fill then covers the halos only.  A first stage without
    // that output (after a state change or a download of W) fills all cells.
    const bool w_ready = ctx->fused_ready && ctx->w_next_ready;
    NS_TRY(exchange(ctx, NS_EXCHANGE_DT, nullptr, cur));
    for (int st = 0; st < 3; st++) {
        NS_TRY(exchange(ctx, NS_EXCHANGE_HALO, in[st], nullptr));
        if (st == 0 && !w_ready)
            launch_fill_prim(ctx->W, in[st], ctx->box, ctx->c, s, out[st]);
        else
            launch_fill_halo(ctx->W, in[st], ctx->box, ctx->c, s, out[st]);
        NS_TRY(check_launch(ctx, 1));
        prof_mark(ctx, NS_PROF_FILL);
        NS_TRY(xstage(ctx, st, in[st], out[st], cur, nxt, true, Planes()));
        std::swap(ctx->W, ctx->W2);
    }
    end_xstep(ctx);
    return NS_OK;
}

// W = prim(U) on every cell after a step.  After fused steps U's ghost cells
// are stale, so they are refilled from the interior first (the interior is what
// the reference's W holds; its ghost cells then hold the filled values).
static ns_status finalize_w(ns_ctx* ctx) {
    if (!ctx->w_valid) {
        ctx->w_next_ready = false;  // W is about to hold prim(U), not the next stage's W
        if (ctx->halos_stale)
            launch_fill_prim(ctx->W, ctx->U, ctx->box, ctx->c, ctx->stream);
        else
            launch_prim_all(ctx->W, ctx->U, ctx->box, ctx->c, ctx->stream);
        NS_TRY(check_launch(ctx, 1));
        ctx->w_valid = true;
        ctx->halos_stale = false;
    }
    return NS_OK;
}

// params.check_finite: counts the interior cells of the current state that hold
// NaN/Inf or a non-positive density or pressure (waits for the stream)
static ns_status check_state(ns_ctx* ctx) {
    if (!ctx->p.check_finite || (!ctx->w_valid && !ctx->u_valid)) return NS_OK;
    cudaStream_t s = ctx->stream;
    unsigned long long* cnt = ctx->slot + 3;
    NS_CUDA(cudaMemsetAsync(cnt, 0, sizeof *cnt, s));
    if (ctx->u_valid) launch_check_state(ctx->U, false, ctx->box, ctx->c, cnt, s);
    else launch_check_state(ctx->W, true, ctx->box, ctx->c, cnt, s);
    NS_TRY(check_launch(ctx, 1));
    unsigned long long n = 0;
    NS_CUDA(cudaMemcpyAsync(&n, cnt, sizeof n, cudaMemcpyDeviceToHost, s));
    NS_CUDA(cudaStreamSynchronize(s));
    if (n)
        return fail(NS_ERR_NONFINITE,
                    "%llu interior cells hold NaN/Inf or a non-positive density or pressure after %lld steps",
                    n, ctx->steps);
    return NS_OK;
}

static double slot_dt(unsigned long long bits, double cfl) {
    double v;
    memcpy(&v, &bits, sizeof v);
    return fmin(1e10, v) * cfl;
}

// ===========================================================================
extern "C" {

const char* ns_status_string(ns_status s) {
    switch (s) {
        case NS_OK: return "ok";
        case NS_ERR_INVALID_ARG: return "invalid argument";
        case NS_ERR_OOM: return "out of device memory";
        case NS_ERR_CUDA: return "CUDA error";
        case NS_ERR_NONFINITE: return "non-finite state";
        case NS_ERR_TIMEOUT: return "device wait timed out";
        case NS_ERR_UNSUPPORTED: return "unsupported";
        case NS_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

const char* ns_last_error_string(void) { return g_err.c_str(); }

int ns_abi_version(void) { return NS_ABI_VERSION; }

size_t ns_host_array_elems(const ns_params* p) { return p ? host_elems(p) : 0; }

ns_status ns_params_default(ns_params* p) {
    if (!p) return fail(NS_ERR_INVALID_ARG, "params is NULL");
    memset(p, 0, sizeof *p);
    // tutorials/shearLayer/input.xml values, 3D
    p->dim = 3;
    p->nx = p->ny = p->nz = 64;
    p->Lx = p->Ly = p->Lz = 1.0;
    p->mu = 1e-4;
    p->Pr = 0.71;
    p->gamma = 1.4;
    p->cfl = 0.4;
    p->convection = NS_CONV_WENO5;
    p->weights = NS_WEIGHTS_SHU;
    p->diffusion = NS_DIFF_CENTERED;
    p->diffusion_order = 2;
    p->bc[0] = p->bc[1] = p->bc[2] = NS_BC_PERIODIC;
    p->precision = NS_PREC_FP64;
    p->semantics = NS_SEM_REFERENCE;
    p->sensor = 0;
    p->sensor_threshold = 0.5;
    return NS_OK;
}

void ns_destroy(ns_ctx* ctx) {
    if (!ctx) return;
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->W);
    cudaFree(ctx->U);
    cudaFree(ctx->U0);
    cudaFree(ctx->U2);
    cudaFree(ctx->W2);
    cudaFree(ctx->R);
    for (int d = 0; d < 3; d++) cudaFree(ctx->F[d]);
    cudaFree(ctx->stage);
    cudaFree(ctx->slot);
    cudaFree(ctx->diag);
    cudaFree(ctx->clock);
    if (ctx->sensor) sensor_destroy(ctx->sensor);
    if (ctx->copy) {
        cudaStreamSynchronize(ctx->copy);
        cudaStreamDestroy(ctx->copy);
    }
    for (cudaEvent_t e : ctx->ev) cudaEventDestroy(e);
    if (ctx->own) cudaStreamDestroy(ctx->own);
    delete ctx;
}

ns_status ns_create(const ns_params* p, ns_ctx** out) {
    if (!out) return fail(NS_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    NS_TRY(validate(p));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(NS_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    ns_ctx* ctx = new (std::nothrow) ns_ctx();
    if (!ctx) return fail(NS_ERR_OOM, "host allocation failed");
    ctx->p = *p;
    ctx->box = make_box(p->nx, p->ny, p->nz);
    for (int d = 0; d < 3; d++) ctx->fb[d] = make_facebox(p->nx, p->ny, p->nz, d);
    ctx->c = make_consts(p);
    cudaGetDevice(&ctx->device);
    cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, ctx->device);
    ns_status st = NS_OK;
    auto A = [&](void** ptr, size_t bytes) {
        if (st != NS_OK) return;
        cudaError_t e = cudaMalloc(ptr, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            st = fail(e == cudaErrorMemoryAllocation ? NS_ERR_OOM : NS_ERR_CUDA,
                      "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
        }
    };
    if (cudaStreamCreateWithFlags(&ctx->own, cudaStreamNonBlocking) != cudaSuccess) {
        ns_destroy(ctx);
        return fail(NS_ERR_CUDA, "cudaStreamCreate failed");
    }
    ctx->stream = ctx->own;
    A((void**)&ctx->W, soa_bytes(ctx->box));
    A((void**)&ctx->U, soa_bytes(ctx->box));
    A((void**)&ctx->U0, soa_bytes(ctx->box));
    size_t fe = fp32(ctx) ? sizeof(float) : sizeof(double);
    if (p->convection != NS_CONV_NONE)
        for (int d = 0; d < (p->dim == 3 ? 3 : 2); d++)
            A(&ctx->F[d], (size_t)ctx->fb[d].fstride * NS_NQ * fe);
    // [0], [1]: CFL minima by step parity, [2]: scratch minimum, [3]: count of
    // bad cells (check_finite), [4]: error word of the bounded device waits
    A((void**)&ctx->slot, 5 * sizeof(unsigned long long));
    // The fused stage kernel serves the FP32 form (both semantics).  In FP64 the
    // face kernels + x-march run faster: an FP64 fused stage on an 8 x 16 column
    // (two 109 KB blocks per SM) measured 1.25-1.56x slower on B200 at 256^3.
    ctx->fused = p->precision == NS_PREC_FP32;
    ctx->xfused = !ctx->fused && p->precision == NS_PREC_FP64 && p->convection != NS_CONV_NONE;
    if (ctx->fused || ctx->xfused) A((void**)&ctx->U2, soa_bytes(ctx->box));
    if (ctx->xfused) A((void**)&ctx->W2, soa_bytes(ctx->box));
    if (st == NS_OK && ctx->xfused) {
        // the y/z faces of the FP64 steps read W (and W2, which swaps with it) through TMA tiles
        nsb::w_tma_encode(&ctx->tma[0], ctx->W, ctx->box);
        nsb::w_tma_encode(&ctx->tma[1], ctx->W2, ctx->box);
    }
    A((void**)&ctx->diag, 8 * sizeof(double));
    A((void**)&ctx->clock, 2 * sizeof(double));
    if (st == NS_OK) {
        // zero the state so halos/corners hold defined values before the first upload
        cudaMemsetAsync(ctx->W, 0, soa_bytes(ctx->box), ctx->stream);
        cudaMemsetAsync(ctx->U, 0, soa_bytes(ctx->box), ctx->stream);
        cudaMemsetAsync(ctx->U0, 0, soa_bytes(ctx->box), ctx->stream);
        cudaMemsetAsync(ctx->clock, 0, 2 * sizeof(double), ctx->stream);
        cudaMemsetAsync(ctx->slot, 0, 5 * sizeof(unsigned long long), ctx->stream);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess)
            st = fail(NS_ERR_CUDA, "initialisation failed: %s", cudaGetErrorString(cudaGetLastError()));
    }
    if (st == NS_OK && p->sensor) st = sensor_create(&ctx->sensor, ctx->box, ctx->fb, ctx->stream);
    if (st != NS_OK) {
        ns_destroy(ctx);
        return st;
    }
    *out = ctx;
    return NS_OK;
}

ns_status ns_set_stream(ns_ctx* ctx, void* stream) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    cudaStream_t s = stream ? (cudaStream_t)stream : ctx->own;
    if (s != ctx->stream) {
        // order the new stream after everything queued on the old one
        cudaEvent_t ev;
        NS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        NS_CUDA(cudaEventRecord(ev, ctx->stream));
        NS_CUDA(cudaStreamWaitEvent(s, ev, 0));
        cudaEventDestroy(ev);
        ctx->stream = s;
    }
    return NS_OK;
}

ns_status ns_upload_primitive(ns_ctx* ctx, const double* W) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    NS_TRY(upload(ctx, W, ctx->W));
    ctx->w_valid = true;
    ctx->u_valid = false;
    ctx->fused_ready = false;
    ctx->flags_valid = false;
    ctx->halos_stale = false;
    NS_CUDA(cudaStreamSynchronize(ctx->stream));
    return NS_OK;
}

ns_status ns_download_primitive(ns_ctx* ctx, double* W) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (!ctx->w_valid && !ctx->u_valid) return fail(NS_ERR_INVALID_ARG, "no state has been uploaded");
    NS_TRY(finalize_w(ctx));
    return download(ctx, ctx->W, W);
}

ns_status ns_download_conservative(ns_ctx* ctx, double* U) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (!ctx->u_valid) return fail(NS_ERR_INVALID_ARG, "no conservative state yet (take a step first)");
    NS_TRY(finalize_w(ctx));
    return download(ctx, ctx->U, U);
}

ns_status ns_convection_solve(ns_ctx* ctx, const double* W, const double* U, double* R) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (!W || !U || !R) return fail(NS_ERR_INVALID_ARG, "W, U and R must be non-NULL");
    NS_TRY(ensure_R(ctx));
    NS_TRY(upload(ctx, W, ctx->W));
    NS_TRY(upload(ctx, U, ctx->U));
    NS_TRY(upload(ctx, R, ctx->R));
    ctx->w_valid = ctx->u_valid = false;  // the device state now holds the operator's inputs
    ctx->fused_ready = ctx->halos_stale = false;
    ctx->flags_valid = false;
    NS_TRY(faces(ctx));
    UpdateArgs a = update_args(ctx, MODE_RHS, true, false);
    launch_update(a, ctx->stream);
    NS_TRY(check_launch(ctx, 1));
    return download(ctx, ctx->R, R);
}

ns_status ns_diffusion_solve(ns_ctx* ctx, const double* W, double* R) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (!W || !R) return fail(NS_ERR_INVALID_ARG, "W and R must be non-NULL");
    NS_TRY(ensure_R(ctx));
    NS_TRY(upload(ctx, W, ctx->W));
    NS_TRY(upload(ctx, R, ctx->R));
    ctx->w_valid = ctx->u_valid = false;
    ctx->fused_ready = ctx->halos_stale = false;
    ctx->flags_valid = false;
    UpdateArgs a = update_args(ctx, MODE_RHS, false, true);
    launch_update(a, ctx->stream);
    NS_TRY(check_launch(ctx, 1));
    return download(ctx, ctx->R, R);
}

ns_status ns_rhs(ns_ctx* ctx, const double* W, double* R, int terms) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (!W || !R) return fail(NS_ERR_INVALID_ARG, "W and R must be non-NULL");
    if (terms < 0 || terms > NS_TERM_ALL) return fail(NS_ERR_INVALID_ARG, "terms must be a mask of NS_TERM_*");
    NS_TRY(ensure_R(ctx));
    NS_TRY(upload(ctx, W, ctx->W));
    NS_TRY(upload(ctx, R, ctx->R));
    cudaStream_t s = ctx->stream;
    ctx->fused_ready = ctx->halos_stale = false;
    ctx->flags_valid = false;
    NS_CUDA(cudaMemsetAsync(ctx->slot + 2, 0xFF, sizeof(unsigned long long), s));
    launch_step_begin(false, phys(ctx), ctx->W, ctx->U, ctx->U0, ctx->box, ctx->c, ctx->slot + 2, s);
    launch_fill_prim(ctx->W, ctx->U, ctx->box, ctx->c, s);
    NS_TRY(check_launch(ctx, 2));
    if (terms & NS_TERM_CONVECTION) NS_TRY(faces(ctx));
    UpdateArgs a = update_args(ctx, MODE_RHS, terms & NS_TERM_CONVECTION, terms & NS_TERM_DIFFUSION);
    a.flags |= UPD_OVERWRITE;
    launch_update(a, s);
    NS_TRY(check_launch(ctx, 1));
    ctx->w_valid = ctx->u_valid = false;
    return download(ctx, ctx->R, R);
}

ns_status ns_compute_dt(ns_ctx* ctx, const double* W, double* dt_out) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (!dt_out) return fail(NS_ERR_INVALID_ARG, "dt_out is NULL");
    NS_TRY(upload(ctx, W, ctx->W));
    ctx->w_valid = true;
    ctx->u_valid = false;
    ctx->fused_ready = ctx->halos_stale = false;
    ctx->flags_valid = false;
    NS_CUDA(cudaMemsetAsync(ctx->slot + 2, 0xFF, sizeof(unsigned long long), ctx->stream));
    launch_min_dt(phys(ctx), ctx->W, ctx->box, ctx->c, ctx->slot + 2, ctx->stream);
    NS_TRY(check_launch(ctx, 1));
    unsigned long long bits;
    NS_CUDA(cudaMemcpyAsync(&bits, ctx->slot + 2, sizeof bits, cudaMemcpyDeviceToHost, ctx->stream));
    NS_CUDA(cudaStreamSynchronize(ctx->stream));
    *dt_out = slot_dt(bits, ctx->p.cfl);
    return NS_OK;
}

static ns_status device_status(ns_ctx* ctx);

#ifndef NS_STEP_PIPELINE
#define NS_STEP_PIPELINE 1  // ns_time_step overlaps its host transfers with the stages
#endif

// x-planes per chunk of ns_time_step's transfer pipeline: whole marches of the
// TMA viscous kernel and of the TMA x-march
static int pipe_chunk() { return std::max(xmarch_planes(), viscous_march_planes()); }

static bool pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// whether ns_time_step runs time_step_pipelined: an FP64 step of do_step's
// x-march form whose kernels all take plane ranges (TMA maps of both W
// buffers), on a single domain, at least two chunks long, from and to pinned
// host memory (to pageable memory a copy blocks the calling thread and
// serialises the chunks)
static bool pipelined(const ns_ctx* ctx, const double* W, const double* U) {
    const ns_params& p = ctx->p;
    if (!NS_STEP_PIPELINE || !NS_XUPD_TMA || !ctx->xfused || ctx->fused || slab(ctx) || p.sensor) return false;
    if (!ctx->tma[0].ok || !ctx->tma[1].ok || p.nx < 2 * pipe_chunk()) return false;
    if (p.diffusion == NS_DIFF_CENTERED && (ctx->c.order > NS_VISC_TMA_MAX_ORDER || !(phys(ctx) || NS_VISC_TMA_REF)))
        return false;
    return pinned(W) && (!U || pinned(U));
}

static ns_status ensure_pipe(ns_ctx* ctx, int nev) {
    if (!ctx->copy) NS_CUDA(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
    while ((int)ctx->ev.size() < nev) {
        cudaEvent_t e;
        NS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->ev.push_back(e);
    }
    return NS_OK;
}

// ns_time_step's upload, do_step and finalize_w + download of W with the host
// transfers overlapped.  W arrives in chunks of x-planes on the copy stream,
// and the first stage's per-plane work (layout transpose, U = cons(W) with the
// step's CFL minimum, the face halos along y and z, W = prim(U), the y- and
// z-face fluxes) runs on each chunk as it lands; the third stage runs chunk by
// chunk (faces, viscous terms, x-march, W = prim(U), layout transpose) and each
// finished chunk of W leaves on the copy stream while the next one computes.
// The kernels and their per-cell arithmetic are those of the unpipelined
// step, so the result is bit-identical.
static ns_status time_step_pipelined_run(ns_ctx* ctx, const double* Wh, double* Wout) {
    const ns_params& p = ctx->p;
    cudaStream_t s = ctx->stream, cs = ctx->copy;
    const int C = pipe_chunk(), nx = p.nx, K = (nx + C - 1) / C;
    cudaEvent_t* ev = ctx->ev.data();  // [0, K) uploads, [K, 2K) downloads, [2K] start, [2K+1] end
    const size_t plane = (size_t)(p.ny + 2 * NS_NGC) * (p.nz + 2 * NS_NGC) * NS_NQ;  // doubles per AoS x-plane
    // chunk c: interior planes [c C, min((c + 1) C, nx)); its halo'd span adds the
    // x ghost planes to the first and the last chunk
    auto interior = [&](int c) {
        Planes pl;
        pl.lo = c * C;
        pl.n = std::min(C, nx - c * C);
        return pl;
    };
    auto halo_interior = [&](int c) {
        Planes pl = interior(c);
        pl.lo += NG;
        return pl;
    };
    auto span = [&](int c) {
        Planes pl;
        pl.lo = c == 0 ? 0 : c * C + NG;
        const int hi = c == K - 1 ? nx + 2 * NG : (c + 1) * C + NG;
        pl.n = hi - pl.lo;
        return pl;
    };
    Planes ghost_lo, ghost_hi;
    ghost_lo.lo = 0;
    ghost_lo.n = NG;
    ghost_hi.lo = nx + NG;
    ghost_hi.n = NG;

    // upload: the copy stream follows the compute stream's earlier use of the staging buffer
    NS_CUDA(cudaEventRecord(ev[2 * K], s));
    NS_CUDA(cudaStreamWaitEvent(cs, ev[2 * K], 0));
    for (int c = 0; c < K; c++) {
        const Planes sp = span(c);
        NS_CUDA(cudaMemcpyAsync(ctx->stage + sp.lo * plane, Wh + sp.lo * plane, sp.n * plane * sizeof(double),
                                cudaMemcpyHostToDevice, cs));
        NS_CUDA(cudaEventRecord(ev[c], cs));
    }
    ctx->w_valid = true;
    ctx->u_valid = false;
    ctx->fused_ready = ctx->halos_stale = false;
    ctx->flags_valid = false;
    unsigned long long* cur = ctx->slot + ctx->parity;
    unsigned long long* nxt = ctx->slot + (ctx->parity ^ 1);
    NS_CUDA(cudaMemsetAsync(cur, 0xFF, sizeof(unsigned long long), s));
    NS_CUDA(cudaMemsetAsync(nxt, 0xFF, sizeof(unsigned long long), s));

    // stage 1 (U0 -> U): per chunk as it lands
    for (int c = 0; c < K; c++) {
        const Planes sp = span(c);
        NS_CUDA(cudaStreamWaitEvent(s, ev[c], 0));
        launch_aos_to_soa(ctx->stage, ctx->W, ctx->box, s, sp);
        launch_step_begin(false, phys(ctx), ctx->W, ctx->U, ctx->U0, ctx->box, ctx->c, cur, s, sp);
        launch_fill_prim(ctx->W, ctx->U0, ctx->box, ctx->c, s, ctx->U, halo_interior(c));
        NS_TRY(check_launch(ctx, 3));
        NS_TRY(faces(ctx, 1, ctx->U0, true, interior(c)));
    }
    // the x ghost planes fold onto planes of other chunks
    launch_fill_prim(ctx->W, ctx->U0, ctx->box, ctx->c, s, ctx->U, ghost_lo);
    launch_fill_prim(ctx->W, ctx->U0, ctx->box, ctx->c, s, ctx->U, ghost_hi);
    NS_TRY(check_launch(ctx, 2));
    NS_TRY(xstage(ctx, 0, ctx->U0, ctx->U, cur, nxt, false, Planes()));
    std::swap(ctx->W, ctx->W2);

    // stage 2 (U -> U2)
    launch_fill_halo(ctx->W, ctx->U, ctx->box, ctx->c, s, ctx->U2);
    NS_TRY(check_launch(ctx, 1));
    NS_TRY(xstage(ctx, 1, ctx->U, ctx->U2, cur, nxt, true, Planes()));
    std::swap(ctx->W, ctx->W2);

    // stage 3 (U2 -> U) chunk by chunk into W2, which then holds prim(U) on every
    // cell (finalize_w); U's ghost cells are final after the fill
    launch_fill_halo(ctx->W, ctx->U2, ctx->box, ctx->c, s, ctx->U);
    launch_prim_all(ctx->W2, ctx->U, ctx->box, ctx->c, s, ghost_lo);
    launch_prim_all(ctx->W2, ctx->U, ctx->box, ctx->c, s, ghost_hi);
    NS_TRY(check_launch(ctx, 3));
    for (int c = 0; c < K; c++) {
        NS_TRY(xstage(ctx, 2, ctx->U2, ctx->U, cur, nxt, true, interior(c)));
        const Planes sp = span(c);
        launch_prim_all(ctx->W2, ctx->U, ctx->box, ctx->c, s, halo_interior(c));
        launch_soa_to_aos(ctx->W2, ctx->stage, ctx->box, s, sp);
        NS_TRY(check_launch(ctx, 2));
        NS_CUDA(cudaEventRecord(ev[K + c], s));
        NS_CUDA(cudaStreamWaitEvent(cs, ev[K + c], 0));
        NS_CUDA(cudaMemcpyAsync(Wout + sp.lo * plane, ctx->stage + sp.lo * plane, sp.n * plane * sizeof(double),
                                cudaMemcpyDeviceToHost, cs));
    }
    // the compute stream's next use of the staging buffer follows the downloads
    NS_CUDA(cudaEventRecord(ev[2 * K + 1], cs));
    NS_CUDA(cudaStreamWaitEvent(s, ev[2 * K + 1], 0));
    std::swap(ctx->W, ctx->W2);
    end_xstep(ctx);
    ctx->w_next_ready = false;  // W holds prim(U) (finalize_w)
    ctx->w_valid = true;
    ctx->halos_stale = false;
    NS_CUDA(cudaStreamSynchronize(s));
    return NS_OK;
}

static ns_status time_step_pipelined(ns_ctx* ctx, double* W) {
    NS_TRY(ensure_stage(ctx));
    NS_TRY(ensure_pipe(ctx, 2 * ((ctx->p.nx + pipe_chunk() - 1) / pipe_chunk()) + 2));
    ns_status st = time_step_pipelined_run(ctx, W, W);
    if (st != NS_OK) {
        // no copy of the caller's array may outlive the call
        cudaStreamSynchronize(ctx->copy);
        cudaStreamSynchronize(ctx->stream);
        ctx->w_valid = ctx->u_valid = false;
    }
    return st;
}

ns_status ns_time_step(ns_ctx* ctx, double* W, double* U, double* dt_out) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (!W) return fail(NS_ERR_INVALID_ARG, "W is NULL");
    if (pipelined(ctx, W, U)) {
        NS_TRY(time_step_pipelined(ctx, W));
        double clk[2];
        NS_CUDA(cudaMemcpyAsync(clk, ctx->clock, sizeof clk, cudaMemcpyDeviceToHost, ctx->stream));
        if (U) NS_TRY(download(ctx, ctx->U, U));
        NS_CUDA(cudaStreamSynchronize(ctx->stream));
        if (dt_out) *dt_out = clk[0];
        NS_TRY(device_status(ctx));
        return check_state(ctx);
    }
    NS_TRY(upload(ctx, W, ctx->W));
    ctx->w_valid = true;
    ctx->u_valid = false;
    ctx->fused_ready = ctx->halos_stale = false;
    ctx->flags_valid = false;
    NS_TRY(do_step(ctx));
    NS_TRY(finalize_w(ctx));
    double clk[2];
    NS_CUDA(cudaMemcpyAsync(clk, ctx->clock, sizeof clk, cudaMemcpyDeviceToHost, ctx->stream));
    NS_TRY(download(ctx, ctx->W, W));
    if (U) NS_TRY(download(ctx, ctx->U, U));
    if (dt_out) *dt_out = clk[0];
    NS_TRY(device_status(ctx));
    return check_state(ctx);
}

ns_status ns_host_register(void* ptr, size_t bytes) {
    if (!ptr || bytes == 0) return fail(NS_ERR_INVALID_ARG, "ptr is NULL or bytes is 0");
    NS_CUDA(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
    return NS_OK;
}

ns_status ns_host_unregister(void* ptr) {
    if (!ptr) return fail(NS_ERR_INVALID_ARG, "ptr is NULL");
    NS_CUDA(cudaHostUnregister(ptr));
    return NS_OK;
}

ns_status ns_advance(ns_ctx* ctx, int nsteps) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (nsteps < 0) return fail(NS_ERR_INVALID_ARG, "nsteps must be >= 0");
    if (!ctx->w_valid && !ctx->u_valid) return fail(NS_ERR_INVALID_ARG, "no state has been uploaded");
    for (int n = 0; n < nsteps; n++) NS_TRY(do_step(ctx));
    return check_state(ctx);
}

ns_status ns_get_dt(ns_ctx* ctx, double* dt, double* time) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    double h[2] = {0.0, 0.0};
    NS_CUDA(cudaMemcpyAsync(h, ctx->clock, sizeof h, cudaMemcpyDeviceToHost, ctx->stream));
    NS_CUDA(cudaStreamSynchronize(ctx->stream));
    if (dt) *dt = h[0];
    if (time) *time = h[1];
    return NS_OK;
}

// the status words of the device's bounded waits and self-checks (after the
// stream is idle)
static ns_status device_status(ns_ctx* ctx) {
    if (ctx->sensor && sensor_status(ctx->sensor) != NS_OK)
        return fail(NS_ERR_TIMEOUT, "a tensor-core wait of the sensor's flag kernel ran out of polls");
    unsigned long long werr = 0;
    NS_CUDA(cudaMemcpy(&werr, ctx->slot + 4, sizeof werr, cudaMemcpyDeviceToHost));
    if (werr & 2) return fail(NS_ERR_CUDA, "a TMA kernel found its shared-memory ring misaligned and did nothing");
    if (werr) return fail(NS_ERR_TIMEOUT, "a TMA tile wait of a face, x-march or viscous kernel ran out of polls");
    return NS_OK;
}

ns_status ns_synchronize(ns_ctx* ctx) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    NS_CUDA(cudaStreamSynchronize(ctx->stream));
    NS_TRY(device_status(ctx));
    return check_state(ctx);
}

ns_status ns_get_diagnostics(ns_ctx* ctx, ns_diagnostics* out) {
    if (!ctx || !out) return fail(NS_ERR_INVALID_ARG, "ctx and out must be non-NULL");
    memset(out, 0, sizeof *out);
    out->steps = ctx->steps;
    if (!ctx->w_valid && !ctx->u_valid) return NS_OK;
    cudaStream_t s = ctx->stream;
    NS_TRY(finalize_w(ctx));
    if (!ctx->u_valid) {
        // conservative view of an uploaded primitive state (no step taken yet)
        launch_cons_all(ctx->W, ctx->U, ctx->box, ctx->c, s);
        NS_TRY(check_launch(ctx, 1));
        ctx->u_valid = true;
    }
    NS_CUDA(cudaMemsetAsync(ctx->diag, 0, 8 * sizeof(double), s));
    launch_diagnostics(ctx->U, ctx->box, ctx->c, ctx->diag, s);
    NS_CUDA(cudaMemsetAsync(ctx->slot + 2, 0xFF, sizeof(unsigned long long), s));
    launch_min_dt(phys(ctx), ctx->W, ctx->box, ctx->c, ctx->slot + 2, s);
    NS_TRY(check_launch(ctx, 2));
    double h[8], clk[2];
    unsigned long long bits[3];
    NS_CUDA(cudaMemcpyAsync(h, ctx->diag, sizeof h, cudaMemcpyDeviceToHost, s));
    NS_CUDA(cudaMemcpyAsync(clk, ctx->clock, sizeof clk, cudaMemcpyDeviceToHost, s));
    NS_CUDA(cudaMemcpyAsync(bits, ctx->slot, sizeof bits, cudaMemcpyDeviceToHost, s));
    NS_CUDA(cudaStreamSynchronize(s));
    out->dt = clk[0];
    out->time = clk[1];
    out->next_dt = slot_dt(bits[2], ctx->p.cfl);
    out->mass = h[0];
    out->momentum[0] = h[1];
    out->momentum[1] = h[2];
    out->momentum[2] = h[3];
    out->energy = h[4];
    out->kinetic = h[5];
    out->enstrophy = h[6];
    out->nonfinite = h[7] > 0 ? 1 : 0;
    out->sensor_fraction = ctx->sensor ? sensor_last_fraction(ctx->sensor) : 0.0;
    return NS_OK;
}

ns_status ns_profile_step(ns_ctx* ctx, float* ms, int n) {
    if (!ctx || !ms || n < 7) return fail(NS_ERR_INVALID_ARG, "ctx/ms invalid or n < 7");
    if (!ctx->w_valid && !ctx->u_valid) return fail(NS_ERR_INVALID_ARG, "no state has been uploaded");
    Prof pr;
    for (int e = 0; e < 64; e++) NS_CUDA(cudaEventCreate(&pr.ev[e]));
    cudaEvent_t start;
    NS_CUDA(cudaEventCreate(&start));
    NS_CUDA(cudaEventRecord(start, ctx->stream));
    g_prof = &pr;
    ns_status st = do_step(ctx);
    g_prof = nullptr;
    if (st == NS_OK) st = (cudaStreamSynchronize(ctx->stream) == cudaSuccess)
                              ? NS_OK : fail(NS_ERR_CUDA, "profiled step failed");
    for (int c = 0; c < n; c++) ms[c] = 0.f;
    cudaEvent_t prev = start;
    for (int e = 0; e < pr.n && st == NS_OK; e++) {
        float t = 0.f;
        cudaEventElapsedTime(&t, prev, pr.ev[e]);
        if (pr.cls[e] < n) ms[pr.cls[e]] += t;
        prev = pr.ev[e];
    }
    for (int e = 0; e < 64; e++) cudaEventDestroy(pr.ev[e]);
    cudaEventDestroy(start);
    return st;
}

long long ns_kernel_launches(ns_ctx* ctx) { return ctx ? ctx->launches : 0; }

ns_status ns_div_selftest(long long n, unsigned long long seed, unsigned long long* max_ulp) {
    if (!max_ulp || n <= 0) return fail(NS_ERR_INVALID_ARG, "max_ulp must be non-NULL and n positive");
    unsigned long long* d = nullptr;
    NS_CUDA(cudaMalloc(&d, 2 * sizeof *d));
    ns_status st = NS_OK;
    unsigned long long h[2] = {0, 0};
    if (cudaMemset(d, 0, 2 * sizeof *d) != cudaSuccess || launch_div_check(n, seed, d, nullptr) != cudaSuccess ||
        cudaMemcpy(h, d, sizeof h, cudaMemcpyDeviceToHost) != cudaSuccess)
        st = fail(NS_ERR_CUDA, "division self-test failed: %s", cudaGetErrorString(cudaGetLastError()));
    cudaFree(d);
    if (st == NS_OK) {
        max_ulp[0] = h[0];
        max_ulp[1] = h[1];
    }
    return st;
}

ns_status ns_wait_selftest(unsigned polls, int* ran_out, double* ms) {
    if (!ran_out || !ms) return fail(NS_ERR_INVALID_ARG, "ran_out and ms must be non-NULL");
    if (polls == 0 || polls > (1u << 24)) return fail(NS_ERR_INVALID_ARG, "polls must lie in 1 .. 2^24");
    unsigned long long* out = nullptr;
    NS_CUDA(cudaMalloc(&out, sizeof *out));
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ns_status st = NS_OK;
    unsigned long long h = 2;
    float t = 0.f;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess || cudaMemsetAsync(out, 0xFF, sizeof *out, s) != cudaSuccess ||
        cudaEventRecord(e0, s) != cudaSuccess || launch_wait_probe(polls, out, s) != cudaSuccess ||
        cudaEventRecord(e1, s) != cudaSuccess ||
        cudaMemcpyAsync(&h, out, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess || cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
        st = fail(NS_ERR_CUDA, "wait self-test failed: %s", cudaGetErrorString(cudaGetLastError()));
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    cudaFree(out);
    if (st != NS_OK) return st;
    if (h > 1) return fail(NS_ERR_CUDA, "wait self-test wrote no result");
    *ran_out = (int)h;
    *ms = t;
    return NS_OK;
}

ns_status ns_fma_peak(int fp64, double* tflops) {
    if (!tflops) return fail(NS_ERR_INVALID_ARG, "tflops is NULL");
    int dev = 0, sms = 0;
    NS_CUDA(cudaGetDevice(&dev));
    NS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, iters = 4096;
    void* sink = nullptr;
    NS_CUDA(cudaMalloc(&sink, 16));
    cudaStream_t s;
    cudaEvent_t e0, e1;
    NS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    NS_CUDA(cudaEventCreate(&e0));
    NS_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    ns_status st = NS_OK;
    for (int r = 0; r < 5 && st == NS_OK; r++) {
        cudaEventRecord(e0, s);
        if (launch_fma_probe(fp64 != 0, blocks, iters, sink, s) != cudaSuccess)
            st = fail(NS_ERR_CUDA, "FMA probe launch failed");
        cudaEventRecord(e1, s);
        if (cudaEventSynchronize(e1) != cudaSuccess) st = fail(NS_ERR_CUDA, "FMA probe failed");
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (r > 0 && ms < best) best = ms;  // the first run warms up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    cudaFree(sink);
    if (st != NS_OK) return st;
    const double flops = 2.0 * 8.0 * iters * 256.0 * blocks;
    *tflops = flops / (best * 1e-3) / 1e12;
    return NS_OK;
}

ns_status ns_set_sensor_weights(ns_ctx* ctx, const float* w) {
    if (!ctx || !w) return fail(NS_ERR_INVALID_ARG, "ctx and w must be non-NULL");
    if (!ctx->sensor) return fail(NS_ERR_INVALID_ARG, "the context was created without the sensor (params.sensor = 0)");
    if (sensor_set_weights(ctx->sensor, w, ctx->stream) != NS_OK)
        return fail(NS_ERR_CUDA, "uploading the sensor weights failed");
    return NS_OK;
}

ns_status ns_set_exchange(ns_ctx* ctx, ns_exchange_fn fn, void* user) {
    if (!ctx) return fail(NS_ERR_INVALID_ARG, "ctx is NULL");
    if (!slab(ctx)) return fail(NS_ERR_INVALID_ARG, "the context is not a slab (bc[0] != NS_BC_EXTERNAL)");
    ctx->xfn = fn;
    ctx->xuser = user;
    return NS_OK;
}

size_t ns_slab_elems(ns_ctx* ctx) { return ctx ? (size_t)15 * ctx->p.ny * ctx->p.nz : 0; }

ns_status ns_slab_pack(ns_ctx* ctx, int side, void* buf) {
    if (!ctx || !buf || (side != 0 && side != 1)) return fail(NS_ERR_INVALID_ARG, "ctx, side or buffer invalid");
    if (ctx->xwhat != NS_EXCHANGE_HALO || !ctx->xbuf)
        return fail(NS_ERR_INVALID_ARG, "ns_slab_pack is valid inside the NS_EXCHANGE_HALO callback only");
    launch_slab_pack(ctx->xbuf, ctx->box, side, (double*)buf, ctx->stream);
    return check_launch(ctx, 1);
}

ns_status ns_slab_unpack(ns_ctx* ctx, int side, const void* buf) {
    if (!ctx || !buf || (side != 0 && side != 1)) return fail(NS_ERR_INVALID_ARG, "ctx, side or buffer invalid");
    if (ctx->xwhat != NS_EXCHANGE_HALO || !ctx->xbuf)
        return fail(NS_ERR_INVALID_ARG, "ns_slab_unpack is valid inside the NS_EXCHANGE_HALO callback only");
    launch_slab_unpack(ctx->xbuf, ctx->box, side, (const double*)buf, ctx->stream);
    return check_launch(ctx, 1);
}

ns_status ns_slab_dt_slot(ns_ctx* ctx, void** ptr) {
    if (!ctx || !ptr) return fail(NS_ERR_INVALID_ARG, "ctx or ptr is NULL");
    if (ctx->xwhat != NS_EXCHANGE_DT || !ctx->xslot)
        return fail(NS_ERR_INVALID_ARG, "ns_slab_dt_slot is valid inside the NS_EXCHANGE_DT callback only");
    *ptr = ctx->xslot;
    return NS_OK;
}

ns_status ns_sensor_harvest(ns_ctx* ctx, float* feat, float* label, long long capacity, long long* count,
                            double rel_threshold) {
    if (!ctx || !feat || !label || !count) return fail(NS_ERR_INVALID_ARG, "NULL argument");
    if (!ctx->w_valid && !ctx->u_valid) return fail(NS_ERR_INVALID_ARG, "no state has been uploaded");
    if (!(rel_threshold > 0.0)) return fail(NS_ERR_INVALID_ARG, "rel_threshold must be > 0");
    const int nd = ctx->p.dim == 3 ? 3 : 2;
    long long need = 0;
    for (int d = 0; d < nd; d++) need += (long long)ctx->fb[d].n0 * ctx->fb[d].n1 * ctx->fb[d].n2;
    *count = need;
    if (need > capacity)
        return fail(NS_ERR_INVALID_ARG, "harvest needs %lld rows, capacity is %lld", need, capacity);
    cudaStream_t s = ctx->stream;
    // the stage-1 view of the current state: U = cons(W) on all cells, boundary fill, W = prim(U)
    NS_TRY(finalize_w(ctx));
    launch_cons_all(ctx->W, ctx->U, ctx->box, ctx->c, s);
    launch_fill_prim(ctx->W, ctx->U, ctx->box, ctx->c, s);
    NS_TRY(check_launch(ctx, 2));
    ctx->u_valid = true;
    ctx->w_valid = true;
    ctx->halos_stale = false;
    long long base = 0;
    for (int d = 0; d < nd; d++) {
        if (sensor_harvest(d, ctx->p.weights == NS_WEIGHTS_BORGES, phys(ctx), ctx->W, ctx->U, ctx->box, ctx->c,
                           ctx->fb[d], base, rel_threshold, feat, label, s) != NS_OK)
            return fail(NS_ERR_CUDA, "harvest kernel launch failed: %s", cudaGetErrorString(cudaGetLastError()));
        NS_TRY(check_launch(ctx, 1));
        base += (long long)ctx->fb[d].n0 * ctx->fb[d].n1 * ctx->fb[d].n2;
    }
    NS_CUDA(cudaStreamSynchronize(s));
    return NS_OK;
}

}  // extern "C"

// ===========================================================================
// Convection residual without any device allocation.
//
// For callers that must not allocate device memory themselves or have it
// allocated on their behalf: host programs that hand out all device memory
// from their own pool and give a plugin no allocation budget, and control or
// real-time loops that cannot afford cudaMalloc's latency, its implicit device
// synchronisation or an out-of-memory failure in the middle of a run.  The
// caller supplies the inputs and the output in device memory; the face fluxes
// that the other entry points keep in context-owned buffers live here in one
// fixed array compiled into the library.
//
// Cost and limits: the array takes NS_NOALLOC_SCRATCH_BYTES (32 MiB) on every
// GPU where this library's device code is loaded, for the life of the process.
// CUDA loads a library's device code onto a device lazily by default (since
// CUDA 12.2), at the first use of one of its kernels or symbols there, so the
// array may be reserved by the first call of this entry point on a device; a
// caller that must not see an out-of-memory failure later makes one call at
// start-up (or runs with CUDA_MODULE_LOADING=EAGER).  That first call on a
// device also loads the device code, which is not allowed inside a stream
// capture: make it before any capture begins.  A grid fits when the face
// fluxes of all convected axes fit in the array (FP64: 5 doubles per face;
// about 64^3 cells in 3D); larger grids are rejected with NS_ERR_INVALID_ARG.
// All calls on a device share the array, so calls whose kernels overlap on
// that GPU (different streams, or several host threads) race and corrupt each
// other's results; serialise them.  Every scratch element a call reads is
// written earlier in the same call, so nothing needs clearing between calls.
namespace {

constexpr size_t kNoAllocScratchBytes = NS_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

// Device address of the scratch array in the current context.  The symbol's
// host-side name is only a stand-in, so the address is looked up with the
// target device current, on every call: a cached address would go stale when
// the context is destroyed (cudaDeviceReset) or when the caller switches to
// another context on the same device.  The lookup is a host-side table read
// once the device code is loaded.
ns_status noalloc_scratch(void** out) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
        int dev = -1;
        cudaGetDevice(&dev);
        return fail(NS_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed on device %d: %s", dev,
                    cudaGetErrorString(e));
    }
    *out = ptr;
    return NS_OK;
}

}  // namespace

extern "C" ns_status ns_convection_solve_noalloc(const ns_params* p, const double* W,
                                                 const double* U, double* R, void* stream) {
    NS_TRY(validate(p));
    if (!W || !U || !R) return fail(NS_ERR_INVALID_ARG, "W, U and R must be non-NULL device pointers");
    if (p->convection == NS_CONV_NONE)
        return fail(NS_ERR_INVALID_ARG, "convection is NS_CONV_NONE: there is no residual to compute");
    if (p->sensor) return fail(NS_ERR_UNSUPPORTED, "the sensor-gated form needs a context (ns_create)");
    // the caller's layout: 5 planes of the halo'd box, unpadded, k fastest
    Box b;
    b.nx = p->nx; b.ny = p->ny; b.nz = p->nz;
    b.NX = p->nx + 2 * NS_NGC; b.NY = p->ny + 2 * NS_NGC; b.NZp = p->nz + 2 * NS_NGC;
    b.fstride = (long long)b.NX * b.NY * b.NZp;
    FaceBox fb[3];
    for (int d = 0; d < 3; d++) fb[d] = make_facebox(p->nx, p->ny, p->nz, d);
    const int nd = p->dim == 3 ? 3 : 2;
    const bool f32 = p->precision == NS_PREC_FP32;
    const size_t elem = f32 ? sizeof(float) : sizeof(double);
    size_t need = 0;
    for (int d = 0; d < nd; d++) need += (size_t)NS_NQ * (size_t)fb[d].fstride * elem;
    if (need > kNoAllocScratchBytes)
        return fail(NS_ERR_INVALID_ARG,
                    "grid %dx%dx%d needs %zu bytes of face-flux scratch; the no-allocation entry point "
                    "holds %zu bytes (about 64^3 cells in FP64)",
                    p->nx, p->ny, p->nz, need, kNoAllocScratchBytes);
    void* base = nullptr;
    NS_TRY(noalloc_scratch(&base));
    const Consts c = make_consts(p);
    cudaStream_t s = (cudaStream_t)stream;
    void* F[3] = {nullptr, nullptr, nullptr};
    char* cur = (char*)base;
    for (int d = 0; d < nd; d++) {
        F[d] = cur;
        cur += (size_t)NS_NQ * (size_t)fb[d].fstride * elem;
    }
    const bool chr = p->convection == NS_CONV_WENO5_CHAR;
    const bool borges = p->weights == NS_WEIGHTS_BORGES;
    const bool ph = p->semantics == NS_SEM_PHYSICAL;
    for (int d = 0; d < nd; d++) launch_face_flux(d, chr, borges, ph, f32, W, U, b, c, F[d], fb[d], s);
    UpdateArgs a;
    memset(&a, 0, sizeof a);
    a.W = W;
    for (int d = 0; d < 3; d++) { a.F[d] = F[d]; a.fb[d] = fb[d]; }
    a.b = b;
    a.c = c;
    a.flags = UPD_CONV | (p->dim == 3 ? UPD_CONVZ : 0);
    a.mode = MODE_RHS;
    a.viscous = false;
    a.phys = ph;
    a.fp32 = f32;
    a.Rout = R;
    launch_update(a, s);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NS_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
    return NS_OK;
}
