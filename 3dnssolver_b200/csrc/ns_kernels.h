// ns_kernels.h -- host-side launchers of the device kernels (internal).
#pragma once

#include <cuda_runtime.h>

#include "ns_common.cuh"

namespace nsb {

enum { MODE_STAGE = 0, MODE_RHS = 1 };
enum { UPD_CONV = 1, UPD_CONVZ = 2, UPD_OVERWRITE = 4 };

struct UpdateArgs {
    const double* W;
    double* U;
    const double* U0;
    const void* F[3];
    Box b;
    FaceBox fb[3];
    Consts c;
    int flags;       // UPD_*
    int mode;        // MODE_*
    bool viscous;
    bool phys;
    bool fp32;
    const unsigned long long* slot;  // reduced CFL minimum of this step
    double m1, m2, mc;               // U = U0*m1 + U*m2 + R*(mc*dt)
    double* Rout;                    // MODE_RHS target (halo'd SoA)
    double* clock;                   // [last dt, accumulated time], updated once per step (nullable)
    double* Unext;                   // launch_xface_update: the stage's output buffer
    double* Wnext;                   // launch_xface_update: the next stage's W (interior)
    unsigned long long* slot_next;   // launch_xface_update, third stage: the next step's CFL
                                     // minimum (U0 then receives the next step's start)
    const double* V;                 // launch_xface_update with viscous terms: launch_viscous's output
    long long vs;                    // its plane stride
};

// per-face flags of the learned sensor (1 = characteristic-wise), FaceBox order
struct Gate {
    const unsigned char* m[3];
    FaceBox fb[3];
};

// The learned sensor's flags of a step in the form the correction passes read:
// per axis the flag bytes and a compacted list of the flagged faces (FaceBox
// indices), and the cells next to a flagged face (one byte per cell, and a
// compacted list of interior indices (i ny + j) nz + k).  Counts on the device.
struct GateLists {
    const unsigned* face_list[3];
    const unsigned* face_count;  // [3]
    const unsigned* cell_list;
    const unsigned* cell_count;
    const unsigned char* touched;
    const unsigned char* mask[3];
};

// one fused SSP-RK3 stage (ns_fused.cu)
struct FusedArgs {
    const double* Uin;
    double* U0;
    double* Uout;
    Box b;
    Consts c;
    int conv_dims;   // 0 (no convection), 2 or 3
    int visc_h;      // half width of the CD stencil, 0 without diffusion
    bool fp32, chr, borges, last;
    bool phys;                        // physical semantics (local LF speed, textbook eigensystem,
                                      // 3D viscous terms, multi-dimensional CFL)
    double m1, m2, mc;
    const unsigned long long* slot;   // CFL minimum of this step
    unsigned long long* slot_next;    // last stage: CFL minimum of the next step
    double* clock;                    // first stage: [last dt, accumulated time]
    const unsigned char* skip;        // last stage: cells (interior order) whose next-step start a
                                      // correction pass forms instead (nullable)
};
cudaError_t launch_stage_fused(const FusedArgs& a, cudaStream_t s);
// the learned sensor's correction of a fused FP32 stage (ns_gate.cu); F: per-axis
// float face arrays for the flagged faces' flux differences
cudaError_t gate_correct(const FusedArgs& a, const GateLists& L, void* const F[3], const FaceBox fb[3], int sms,
                         cudaStream_t s);

cudaError_t launch_fma_probe(bool fp64, int blocks, int iters, void* sink, cudaStream_t s);

// A range of x-planes [lo, lo + n) for the launchers that take one (n < 0: all
// planes).  The cell kernels (step begin, prim, fill, layout transposes) count
// halo'd planes (0 .. nx+5); the y/z-face, viscous and x-march kernels count
// interior planes (0 .. nx-1), and for the marched kernels (viscous, x-march)
// lo is a multiple of their march length and lo + n is one too or nx.
struct Planes {
    int lo = 0, n = -1;
};
// march lengths along x of the TMA viscous kernel and of the TMA x-march
int viscous_march_planes();
int xmarch_planes();

void launch_step_begin(bool from_u, bool phys, double* W, double* U, double* U0, const Box& b,
                       const Consts& c, unsigned long long* slot, cudaStream_t s, Planes pl = Planes());
void launch_prim_all(double* W, const double* U, const Box& b, const Consts& c, cudaStream_t s,
                     Planes pl = Planes());
void launch_cons_all(const double* W, double* U, const Box& b, const Consts& c, cudaStream_t s);
void launch_min_dt(bool phys, const double* W, const Box& b, const Consts& c, unsigned long long* slot,
                   cudaStream_t s);
// face halos of U and W only (the interior of W is already the stage's)
void launch_fill_halo(double* W, double* U, const Box& b, const Consts& c, cudaStream_t s,
                      double* Uhalo = nullptr);
// Uhalo (nullable) receives the same face-halo values as U
void launch_fill_prim(double* W, double* U, const Box& b, const Consts& c, cudaStream_t s,
                      double* Uhalo = nullptr, Planes pl = Planes());
// w_only (FP64 y- and z-faces of a time step, where W = prim(U)): U = cons(W)
void launch_face_flux(int dir, bool chr, bool borges, bool phys, bool fp32, const double* W,
                      const double* U, const Box& b, const Consts& c, void* F, const FaceBox& fb,
                      cudaStream_t s, bool w_only = false, Planes pl = Planes());
// the last y or z face plane (j = ny or k = nz) of an FP64 time step (W only)
void launch_face_tail_w(int dir, bool chr, bool borges, bool phys, const double* W, const Box& b,
                        const Consts& c, void* F, const FaceBox& fb, cudaStream_t s, Planes pl = Planes());
// TMA tensor maps of one W buffer (ns_tma.cu): map[0] the y-face tiles, map[1]
// the z-face tiles, map[2] the x-march's planes, map[3 + h - 1] the planes of the
// marched viscous kernel of half-width h (CD-2h); each holds a CUtensorMap
// (128 bytes, 64-byte aligned)
struct WTmaMaps {
    alignas(64) unsigned char map[6][128];
    const double* W = nullptr;
    bool ok = false;
};
// one plane of the TMA-marched viscous kernel of half-width H for a block of
// 4 rows x 32 columns (halo'd coordinates): rows j0+3-H .. j0+6+H, columns from
// k0+3-H rounded down to even (TMA's innermost start rule), 32 + 2H (+1) wide
// rounded up to even; lane 0's cell sits in column C0
template <int H>
struct ViscTile {
    static constexpr int Z0 = (3 - H) & ~1;          // box start minus k0
    static constexpr int C0 = 3 - Z0;                // lane 0's cell column in the box
    static constexpr int BZ = (C0 + 32 + H + 1) & ~1;  // columns
    static constexpr int BY = 4 + 2 * H;             // rows
};
// false (and m->ok false) where TMA cannot serve the buffer: no driver entry
// point, an unaligned base or too many tiles; the per-thread kernels then run
bool w_tma_encode(WTmaMaps* m, const double* W, const Box& b);
// FP64 y- (dir 1) or z-faces (dir 2) of a time step from TMA-loaded tiles of the
// W that m maps, then the last face plane; *err receives 1 if a wait ran out
void launch_face_flux_tma(int dir, bool chr, bool borges, bool phys, const WTmaMaps& m, const double* W,
                          const Box& b, const Consts& c, void* F, const FaceBox& fb, int sms,
                          unsigned long long* err, cudaStream_t s, Planes pl = Planes());
// largest ulp distance between div_pos_nr and the IEEE quotient over n draws
cudaError_t launch_div_check(long long n, unsigned long long seed, unsigned long long* max_ulp, cudaStream_t s);
// one block waits (bounded) on an mbarrier phase nothing completes; out[0] = 1
// if the wait gave up, 0 if it claimed completion
cudaError_t launch_wait_probe(unsigned polls, unsigned long long* out, cudaStream_t s);
void launch_update(const UpdateArgs& a, cudaStream_t s);
// FP64 MODE_STAGE: x-faces + update in one march, U_out = a.Unext (a.F[0] unused)
void launch_xface_update(bool chr, bool borges, const UpdateArgs& a, cudaStream_t s);
// the same with the x-stencil's W from TMA-loaded planes of the W that m maps
// (a.W is that W); *err receives 1 if a wait ran out
void launch_xface_update_tma(bool chr, bool borges, const UpdateArgs& a, const WTmaMaps& m, unsigned long long* err,
                             cudaStream_t s, Planes pl = Planes());
// viscous terms (components 1..4) of every interior cell into V (plane stride
// vs >= nx ny nz), half-width h = order/2 of the centered scheme
void launch_viscous(int h, bool phys, const double* W, const Box& b, const Consts& c, double* V,
                    long long vs, cudaStream_t s);
// the same from TMA-loaded planes of the W that m maps, marched along x
// (half-width h = 1, 2, 3); *err receives 1 if a wait ran out
void launch_viscous_tma(int h, bool phys, const WTmaMaps& m, const double* W, const Box& b, const Consts& c,
                        double* V, long long vs, unsigned long long* err, cudaStream_t s, Planes pl = Planes());
// slab halo exchange: pack the outer interior planes of a side / unpack into its ghost planes
void launch_slab_pack(const double* U, const Box& b, int side, double* buf, cudaStream_t s);
void launch_slab_unpack(double* U, const Box& b, int side, const double* buf, cudaStream_t s);
void launch_aos_to_soa(const double* A, double* S, const Box& b, cudaStream_t s, Planes pl = Planes());
void launch_soa_to_aos(const double* S, double* A, const Box& b, cudaStream_t s, Planes pl = Planes());
// interior cells of A (W if prim, else U) that are non-finite or have rho <= 0 or p <= 0,
// added to *count
void launch_check_state(const double* A, bool prim, const Box& b, const Consts& c,
                        unsigned long long* count, cudaStream_t s);
void launch_diagnostics(const double* U, const Box& b, const Consts& c, double* acc, cudaStream_t s);

}  // namespace nsb
