// Internal declarations shared by the kcig sources (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/kcig.h"

namespace kcig {

// ------------------------------------------------------------------ errors --
int set_error(int code, const char *fmt, ...);
// Raises a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device, calling the runtime only when the limit must grow (so a
// launch sequence under stream capture makes no attribute calls once warm);
// carveout >= 0 also sets the kernel's preferred shared-memory carveout then.
int set_dyn_smem(const void *fn, int bytes, int carveout = -1);
int cuda_error(cudaError_t e, const char *what);

#define KCIG_CUDA(call)                                               \
    do {                                                              \
        cudaError_t e__ = (call);                                     \
        if (e__ != cudaSuccess) return ::kcig::cuda_error(e__, #call); \
    } while (0)

#define KCIG_TRY(expr)            \
    do {                          \
        int rc__ = (expr);        \
        if (rc__ != KCIG_OK) return rc__; \
    } while (0)

// Interpolation of one leg (source or receiver) along the table position
// axis, resolved on the host in double precision from the reference's
// branch rules (src/kirchmig2d_cig.cpp:987-1029 and :1148-1180).
struct LegInterp {
    int i0;        // left slice
    int i1;        // right slice, or -1: take slice i0 unchanged (clamped end)
    int type;      // 'h', 'l', 'p'
    int k1, k2;    // 'p' slice shifts (tinterpsr.cpp:86-87)
    double c[4];   // T  = c0*p0 + c1*m0 + c2*p1 + c3*m1
    double e[4];   // Tx = e0*p0 + e1*m0 + e2*p1 + e3*m1
    double t, dxp; // in-interval fraction and position spacing ('p')
    int gi0, gi1;  // gradient-volume slices (interp_volume_linear_stream, :294-322)
    double gw;     // weight of gi1 (0: copy gi0)
    double pos;    // surface position of the leg (aperture)
    float scale;   // ds (source) or dh (receiver): Tx is stored as Tx*scale
    float posf;    // the same position in the reference's float arithmetic
    // kirchmig2d, cmp=1 receiver right of its source: the cone's right-side
    // test is written ((x0 + ix*dx) - s) - h there (:461), so the leg keeps
    // its shot's s and h (cexact = 1) instead of using posf = s + h
    int cexact;
    float cs, ch;
};

// Device views of a batch of leg fields.  The opening angle of a pair is the
// difference of the two legs' gradient directions, so each leg stores the
// polar angle phi = atan2(gz, gx) of its stabilised gradient (FP64, NaN when
// the gradient vanishes) instead of the two components.
struct LegFields {
    double2 *TP;  // [n][nzx] {traveltime T, gradient direction phi}
    float2 *XW;   // [n][nzx] {Tx*scale, aperture leg weight}
};

struct FieldArgs {
    const float *tab, *der;       // [npos][nzx]
    const float *gxv, *gzv;       // gradient volumes or null
    const LegInterp *legs;        // [n] device
    int n, nz, nx;
    float dz, dx, x0;
    int radius, smooth, angle, use_grad;
    float aper, aper_taper, rmin, rtaper;
    int cone;  // kirchmig2d: the w field holds the leg's two cone flags (see k_leg_interp)
    int *status;  // device flag a kernel sets when a bounded wait gives up (may be null)
    int type_p;   // the legs use the partial-shift interpolation ('p')
};

// Workspace for the gradient pipeline: 4 double planes per position.
int launch_leg_fields(const FieldArgs &a, LegFields out, double *work, cudaStream_t st, int *launches = nullptr);
// The two stages of launch_leg_fields: the table interpolation (T, Tx, w;
// with gradient volumes also their interpolation into the work planes), and
// the traveltime gradient of the T already in out.TP -- centred differences
// of radius a.radius, triangle smoothing of radius a.smooth -- into its
// direction phi (out.TP[].y).  launches (if given) is incremented.
int launch_leg_interp(const FieldArgs &a, LegFields out, double *work, cudaStream_t st, int *launches);
int launch_leg_grad(const FieldArgs &a, LegFields out, double *work, cudaStream_t st, int *launches);
// Whether launch_leg_grad uses the work planes (gradient volumes, or a halo
// too wide for the fused kernel): 4 * nzx doubles per leg.
bool leg_grad_needs_work(const FieldArgs &a);

// Leg fields from a traveltime surrogate (kcig_mlp.cu): one launch for all
// `nlegs` legs (only .pos and .scale of each are read).  mode 0: the
// traveltime only (TP[].x; the rest from the tables and the
// finite-difference pass); 1: also its source-position derivative and the
// aperture weight (XW); 2: also the direction phi from the network's own
// input gradient.  The surrogate's status flag is cleared by sg_reset_status
// and read by sg_check_status.
int launch_surrogate_fields(kcig_surrogate *s, const LegInterp *legs, int nlegs, const kcig_geometry &g,
                            const kcig_params &p, LegFields out, int mode, cudaStream_t st);
int sg_reset_status(kcig_surrogate *s, cudaStream_t st);
int sg_check_status(kcig_surrogate *s, cudaStream_t st);

struct PreludeArgs {
    const float *data;      // [ns][nh][nt] whole data cube on the device
    double2 *D;             // [ntr][nt] {D[i], D[i+1]}, ntr = nshots * nhc
    const double *mute_sx;  // [ntr] source x (mute)   (null: no mute)
    const double *mute_rx;  // [ntr] receiver x (mute)
    int ntr, nt, isdiff, invert;
    int nh, nhc, shot0, rcv0;  // batch = shots shot0.., receivers rcv0..rcv0+nhc-1
    double t0, dt, slope, intercept, taper;
    // ragged shots (null for the regular cube): per batch trace, the offset
    // of its samples in `data` (-1: padding, written as zeros) and its
    // sample count (<= nt, the row stride of D)
    const long long *toff;
    const int *tnt;
};
int launch_prelude(const PreludeArgs &a, cudaStream_t st);
int launch_doubint_plain(const float *in, double *out, int ntr, int nt, int isdiff, double dt,
                         cudaStream_t st);

struct SumArgs {
    const double2 *STP;    // [nsb][nzx] source {T, phi}
    const float2 *SXW;     // [nsb][nzx] source {Tx*ds, w}
    const double2 *RTP;    // [nrf][nzx] receiver {T, phi}
    const float2 *RXW;     // [nrf][nzx] receiver {Tx*dh, w}
    const double2 *D;      // [ntr][nt]
    const float *trw;      // [nsb*nh] trace weight, 0 = skip
    const int *rfi;        // [nsb*nh] receiver field index
    const int *igo;        // [nsb*nh] offset-mode bin
    const float *stop;     // [nsb] last usable sample (nt_shot - 1) of ragged shots, or null
    const int *snh;        // [nsb] receivers of each ragged shot (<= nh), or null
    int tile;              // tile variant (kSumTiles), 0 = the default rule
    // the shots of a launch split over `nsplit` CTA rows (grids too small to
    // fill the GPU): row y sums its share into partial[y][ng][nzx], then a
    // fixed-order reduction adds the rows into the image.  nsplit 1: direct.
    int nsplit;
    float *partial;
    float *image;          // [ng][nzx]
    int zero_init;
    int nz, nx, nt, nsb, nh, ng;
    int mode;              // 0 angle two-bin, 1 angle nearest, 2 single bin (offset/stack), 3 kirchmig2d cone + bin
    int unit_tw;           // every trace weight of the batch is 1: trw is not read
    int shared_r;          // receiver fields indexed by ih only (cmp=0)
    int half;
    double t0, dt, inv_dt, tau;
    double deg;            // radians -> output degrees (180/pi, halved for half_angle)
    double ug0, uinv;      // u = (deg*theta - g0) * uinv, the bin coordinate
    float dtf, aal, g0, dg;
    float oazmin, oazmax, oaztaper, ats, ate;
    int gchunk0, gchunk1;  // bin range handled by this launch
};
int launch_sum(const SumArgs &a, cudaStream_t st, int *launches);
// Tile variants the summation can be launched with (the autotuner's choices):
// {TZ, TX, shots per block on the receiver-shared path}.
// Forward modelling (adj=0): the picks of k_sum run backwards, each image
// value sprayed onto the six trace samples of its pick.
struct SprayArgs {
    const double2 *STP;    // [nsb][nzx] source {T, phi}
    const float2 *SXW;     // [nsb][nzx] source {Tx*ds, w}
    const double2 *RTP;    // [nrf][nzx] receiver {T, phi}
    const float2 *RXW;     // [nrf][nzx] receiver {Tx*dh, w}
    const float *trw;      // [nsb*nh] trace weight, 0 = the trace stays zero
    const int *rfi;        // [nsb*nh] receiver field index
    const int *igo;        // [nsb*nh] offset-mode bin
    const float *image;    // [ng][nzx] model
    double *raw;           // [nsb*nh][nt] sprayed traces, before doubint
    int nz, nx, nt, nsb, nh, ng;
    int mode;              // 0 angle two-bin, 1 angle nearest, 2 single bin
    double t0, inv_dt, tau, deg, ug0, uinv;
    float aal, oazmin, oazmax, oaztaper, ats, ate;
};
int launch_spray(const SprayArgs &a, cudaStream_t st);
int launch_doubint_f32(const double *in, float *out, int ntr, int nt, cudaStream_t st);

// How many shot splits a summation over nsb shots on an nz x nx image needs
// to give the GPU at least two waves of CTAs (1: none).
int sum_nsplit(int nz, int nx, int nsb, bool shared_r);
constexpr int kSumTiles = 5;
extern const int kSumTileShape[kSumTiles][3];

}  // namespace kcig
