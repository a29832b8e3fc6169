// K2 + Kf: the NLO part of the BK right-hand side, integrated by quasi-Monte Carlo
// over scrambled Sobol points of the box (log z, log z', theta_z, theta_z') of
// bk/derivatives.py:424-431, with the integrand _nlo_integrand x exp(2 log z + 2 log z')
// of bk/derivatives.py:322-335 and 490-612 (kernels bk_kernels/k2.py:8-39 and
// bk_kernels/kf.py:10-41, coupling at the smallest dipole, RC_NLO = SMALLEST_NLO).
//
// Work decomposition (B200): the points are the same for every parent r, and z,
// z', |z - z'|, their three spline values, the dipole factors of the daughter
// dipoles and the Jacobian do not depend on r.  Each CTA therefore stages a tile
// of samples (one per thread) in shared memory, and every lane then owns one
// active parent and sweeps the whole tile, reading the sample records as
// shared-memory broadcasts.  Per (sample, parent) only X, X', their two spline
// values, the kernels and the coupling remain.  In the mixed build lane sums are FP32
// over 32 samples, folded into FP64 per lane (the FP64 build: compensated sums per
// tile); per-CTA partials go to the caller's workspace and a second kernel adds them in
// a fixed order (deterministic).

#include <cuda_runtime.h>

#include <cstring>
#include <type_traits>

#include "common.cuh"
#include "internal.h"
#include "k2kf_integrand.cuh"
#include "sobol.cuh"

namespace nlo {

namespace {

using namespace k2;

// ---------------------------------------------------------------------------
// FP32 evaluation tuned for instruction count (the kernel is issue-bound).
// Spline values are carried in log2 units; the log S coefficients are stored
// pre-scaled to the unit interval, (a, b h, c h^2, d h^3) * log2(e), so that the
// position u = (log X - x0)/h gives the piece i = floor(u) and t = u - i directly.
// Amplitudes outside the grid are encoded as p2 = 0 (S = 1, below r_min) and
// p2 = -150 (S = 0, above r_max), which lets one branch-free difference formula
// serve every case:  N_A - N_B = S_A (2^(pB-pA) - 1) if pB <= pA, else -S_B (2^(pA-pB) - 1).
__device__ __forceinline__ float ex2_approx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(float x)
{
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}



struct FastSpline {
    // [n + 1] pre-scaled rows (see above): row 0 is (0, 0, 0, 0), the value below r_min
    // (log2 S = 0, S = 1); rows 1..n-1 are the intervals; row n is (-150, 0, 0, 0), above
    // r_max (S = 0)
    const float4* coef;
    float u_scale;  // (ln 2 / 2) / h : u from log2(X^2)
    float u_off;    // -x0 / h
    float u_top;    // n - 1
};

struct P2S {
    float p2, S;
};




struct K2ParentF {
    float r, r2, lr, two_r, four_r;
    float alpha_r;  // the RC_NLO = PARENT_NLO coupling
};

// COUPLING: 0 smooth freeze, 1 smooth freeze capped at alpha_cap, 2 fixed, 3 any coupling
// of alpha_of_log (flavour thresholds), 4 the parent's coupling (RC_NLO = PARENT_NLO).

// Spline position u = (log X - x0)/h -> (log2 S, S) for a pair of positions.  u is clamped
// to [-1, n-1]; the row floor(u) + 1 of the table with its two edge rows serves every case
// (below the grid, inside, above), so there is no edge select.  floor(u) + 1 comes without
// the XU conversions: u + (2^23 + 1) rounded down holds it in the low mantissa bits.  The
// clamp, floor and fraction run on the packed instructions, the table lookup and the cubic
// per component.
__device__ __forceinline__ void fast_amplitude_pair(const FastSpline& s, f2 u, P2S& ax, P2S& ay)
{
    const f2 uc = make_float2(fminf(fmaxf(u.x, -1.0f), s.u_top), fminf(fmaxf(u.y, -1.0f), s.u_top));
    const f2 shifted = __fadd2_rd(uc, bc2(8388609.0f));  // 2^23 + 1 + floor(uc)
    const f2 t = sub2(uc, sub2(shifted, bc2(8388609.0f)));
    const float4 cx = s.coef[__float_as_int(shifted.x) - 0x4B000000];
    const float4 cy = s.coef[__float_as_int(shifted.y) - 0x4B000000];
    const float px = fmaf(t.x, fmaf(t.x, fmaf(t.x, cx.w, cx.z), cx.y), cx.x);
    const float py = fmaf(t.y, fmaf(t.y, fmaf(t.y, cy.w, cy.z), cy.y), cy.x);
    ax = {px, ex2_approx(px)};
    ay = {py, ex2_approx(py)};
}

// ---------------------------------------------------------------------------
// Two samples per call on the packed FP32x2 pipe of sm_100 (FFMA2/FADD2/FMUL2): the
// per-evaluation arithmetic of k2_point_fast, component x for sample 2p and y for 2p+1
// of a pair record (every field of the two samples side by side), so each packed
// instruction does the work of two.  MUFU operations, compares and selects stay scalar.
__device__ __forceinline__ f2 rcp2(f2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }
__device__ __forceinline__ f2 lg22(f2 a) { return make_float2(lg2_approx(a.x), lg2_approx(a.y)); }
__device__ __forceinline__ f2 sel2(bool cx, bool cy, f2 a, f2 b) { return make_float2(cx ? a.x : b.x, cy ? a.y : b.y); }

// N_A - N_B from log2 S values, for a pair
__device__ __forceinline__ f2 fast_ndiff2(const P2S& Ax, const P2S& Ay, const P2S& Bx, const P2S& By)
{
    // N_A - N_B = S_B - S_A.  Near each other (|pB - pA| < 1/2 in log2 units) it is
    // S_A (2^(pB-pA) - 1) or -S_B (2^(pA-pB) - 1) with 2^x - 1 = x q(x), q a degree-5
    // polynomial fitted to (2^x - 1)/x on [-1/2, 0] (1.2e-7 relative in FP32); farther
    // apart the plain difference S_B - S_A has no cancellation (the ratio is at least
    // sqrt(2)), and both S are at hand.
    const f2 d = make_float2(Bx.p2 - Ax.p2, By.p2 - Ay.p2);
    const f2 x = make_float2(-fabsf(d.x), -fabsf(d.y));
    f2 q = fma2(bc2(0.0001327910803141678f), x, bc2(0.001321632968973654f));
    q = fma2(q, x, bc2(0.009615099576281485f));
    q = fma2(q, x, bc2(0.05550375169709732f));
    q = fma2(q, x, bc2(0.24022649146109623f));
    q = fma2(q, x, bc2(0.6931471804499034f));
    const f2 S = make_float2(d.x <= 0.0f ? Ax.S : -Bx.S, d.y <= 0.0f ? Ay.S : -By.S);
    const f2 near = mul2(S, mul2(q, x));
    const f2 far = make_float2(Bx.S - Ax.S, By.S - Ay.S);
    return make_float2(x.x > -0.5f ? near.x : far.x, x.y > -0.5f ? near.y : far.y);
}

template <bool SYM, int COUPLING>
__device__ __forceinline__ void k2_pair_fast(const FastSpline& s, const Phys<float>& ph, const K2ParentF& P,
                                             const float4* __restrict__ rec4, f2& kfw, f2& total)
{
    constexpr float LN2 = 0.69314718055994531f;
    constexpr float L2E = 1.4426950408889634f;
    // pair layout: float4 k holds fields 2k and 2k+1 of (sample x, sample y)
    const float4 w0 = rec4[0], w1 = rec4[1], w2 = rec4[2], w3 = rec4[3], w4 = rec4[4];
    const float4 w5 = rec4[5], w6 = rec4[6], w7 = rec4[7], w8 = rec4[8], w9 = rec4[9];
    const f2 z = make_float2(w0.x, w0.y), z2 = make_float2(w0.z, w0.w);
    const f2 s1 = make_float2(w1.x, w1.y), s2 = make_float2(w1.z, w1.w);
    const f2 P1 = make_float2(w2.x, w2.y), P2 = make_float2(w2.z, w2.w);
    const f2 U1 = make_float2(w3.x, w3.y), V1 = make_float2(w3.z, w3.w);
    const f2 U2 = make_float2(w4.x, w4.y), V2 = make_float2(w4.z, w4.w);
    const f2 q = make_float2(w5.x, w5.y), D1 = make_float2(w5.z, w5.w);
    const f2 D2 = make_float2(w6.x, w6.y), dN = make_float2(w6.z, w6.w);
    const f2 SY = make_float2(w7.x, w7.y), Lmin = make_float2(w7.z, w7.w);
    const f2 cpt = make_float2(w8.x, w8.y), Dl = make_float2(w8.z, w8.w);
    const f2 zsq = make_float2(w9.x, w9.y), z2sq = make_float2(w9.z, w9.w);
    const f2 r = bc2(P.r);
    const f2 rz = sub2(r, z), rz2 = sub2(r, z2);
    const f2 Xsq = fma2(bc2(P.four_r), s1, mul2(rz, rz));  // s1 = z sin^2(theta/2)
    const f2 X2sq = fma2(bc2(P.four_r), s2, mul2(rz2, rz2));
    const f2 L2X = lg22(Xsq), L2X2 = lg22(X2sq);
    const f2 uX = fma2(L2X, bc2(s.u_scale), bc2(s.u_off)), uX2 = fma2(L2X2, bc2(s.u_scale), bc2(s.u_off));
    P2S vXx, vXy, vX2x, vX2y;
    fast_amplitude_pair(s, uX, vXx, vXy);
    fast_amplitude_pair(s, uX2, vX2x, vX2y);
    // kernels
    // log(a/b)/(a - b) = 2 (1 + hm1)/(a + b), hm1 = atanh(t)/t - 1, t = (a - b)/(a + b): the series
    // in t^2 where |a - b| < (a + b)/2, else log(a/b) directly; each case needs one reciprocal,
    // of a + b or of a - b, and the test needs none
    const f2 a = mul2(Xsq, z2sq), b = mul2(X2sq, zsq);
    const f2 sab = add2(a, b);
    const f2 d = mul2(r, fma2(r, P1, make_float2(-P2.x, -P2.y)));  // a - b
    const bool ser_x = fabsf(d.x) < 0.5f * sab.x, ser_y = fabsf(d.y) < 0.5f * sab.y;
    const f2 rden = rcp2(sel2(ser_x, ser_y, sab, d));
    const f2 t = mul2(d, rden);
    const f2 t2 = mul2(t, t);
    f2 g = fma2(bc2(0.15609439065092748f), t2, bc2(0.04106302733766397f));
    g = fma2(g, t2, bc2(0.09747851219255123f));
    g = fma2(g, t2, bc2(0.11051354325642386f));
    g = fma2(g, t2, bc2(0.1428825580061165f));
    g = fma2(g, t2, bc2(0.19999959971627077f));
    g = fma2(g, t2, bc2(0.33333333435159396f));
    const f2 hm1_series = mul2(g, t2);
    const f2 Ld = fma2(bc2(LN2), sub2(L2X, L2X2), Dl);  // log(a/b)
    // log case: 1 + hm1 = log(a/b) (a + b) / (2 (a - b)) and L = log(a/b) / (a - b)
    const f2 Lr = mul2(Ld, rden);
    const f2 hm1 = sel2(ser_x, ser_y, hm1_series, fma2(mul2(bc2(0.5f), Lr), sab, bc2(-1.0f)));
    const f2 rs2 = add2(rden, rden);
    const f2 L = sel2(ser_x, ser_y, fma2(hm1, rs2, rs2), Lr);
    const f2 r2Lq = mul2(mul2(bc2(P.r2), L), q);
    const f2 fq2 = mul2(add2(hm1, hm1), mul2(q, q));
    const f2 C0 = fma2(bc2(-4.0f), r2Lq, fq2);
    const f2 B1 = fma2(r, U1, V1), B2 = fma2(r, U2, V2);
    const f2 w = mul2(r2Lq, bc2(P.two_r));
    const f2 k2 = fma2(mul2(w, B1), rcp2(mul2(Xsq, z2)), C0);
    const f2 k2s = fma2(mul2(w, B2), rcp2(mul2(X2sq, z)), C0);
    const f2 kf = mul2(sub2(r2Lq, fq2), bc2(ph.nf_over_nc));
    const f2 dip = mul2(make_float2(vXx.S, vXy.S), D1), dips = mul2(make_float2(vX2x.S, vX2y.S), D2);
    // the cut |K2| > 1e10 with |dipole| < 1e-10 sets both factors to zero: zero their product
    const bool cut_x = fabsf(k2.x) > 1e10f && fabsf(dip.x) < 1e-10f;
    const bool cut_y = fabsf(k2.y) > 1e10f && fabsf(dip.y) < 1e-10f;
    const f2 prod = sel2(cut_x, cut_y, bc2(0.0f), mul2(k2, dip));
    const f2 dNX = fast_ndiff2(vXx, vXy, vX2x, vX2y);
    f2 k2part, fermion;
    if (SYM) {  // the factor 1/2 of the symmetrisation is folded into cpt
        const bool cuts_x = fabsf(k2s.x) > 1e10f && fabsf(dips.x) < 1e-10f;
        const bool cuts_y = fabsf(k2s.y) > 1e10f && fabsf(dips.y) < 1e-10f;
        k2part = add2(prod, sel2(cuts_x, cuts_y, bc2(0.0f), mul2(k2s, dips)));
        fermion = mul2(mul2(kf, dNX), dN);
    } else {
        k2part = prod;
        fermion = mul2(mul2(kf, SY), dNX);
    }
    f2 alpha;
    if (COUPLING == 2) {
        alpha = bc2(ph.fixed_as);
    } else if (COUPLING == 4) {
        alpha = bc2(P.alpha_r);
    } else {
        const f2 lmin = make_float2(fminf(fminf(Lmin.x, P.lr), (0.5f * LN2) * fminf(L2X.x, L2X2.x)),
                                    fminf(fminf(Lmin.y, P.lr), (0.5f * LN2) * fminf(L2X.y, L2X2.y)));
        if (COUPLING == 3) {
            alpha = make_float2(alpha_of_log(lmin.x, ph), alpha_of_log(lmin.y, ph));
        } else {
            const f2 right = fma2(bc2(-10.0f), lmin, bc2(5.0f * ph.log_sc));
            const f2 m = make_float2(fmaxf(ph.left, right.x), fmaxf(ph.left, right.y));
            const f2 gap = make_float2(fabsf(ph.left - right.x), fabsf(ph.left - right.y));
            // logaddexp = max + log(1 + e^-gap); beyond gap = 17 the correction is below
            // 4.2e-8 of max >= 9.16 (FP32 rounding), and the warp skips the two MUFU operations
            f2 lae = m;
            if (gap.x < 17.0f || gap.y < 17.0f) {
                const f2 e = make_float2(ex2_approx(-gap.x * L2E), ex2_approx(-gap.y * L2E));
                lae = fma2(bc2(LN2), lg22(add2(bc2(1.0f), e)), m);
            }
            alpha = rcp2(mul2(bc2(ph.b0c), lae));
            if (COUPLING == 1) alpha = make_float2(fminf(alpha.x, ph.alpha_cap), fminf(alpha.y, ph.alpha_cap));
        }
    }
    const f2 scale = mul2(mul2(alpha, alpha), cpt);
    const f2 k2w = mul2(k2part, scale);
    kfw = mul2(make_float2(-fermion.x, -fermion.y), scale);
    const f2 tot = add2(k2w, kfw);
    // X^2 or X'^2 below the normal range (the oracle's validity cut) gives infinite kernels
    // (the approximate reciprocal flushes denormals), so the finite test covers it
    const bool ok_x = fabsf(tot.x) < INFINITY;
    const bool ok_y = fabsf(tot.y) < INFINITY;
    kfw = sel2(ok_x, ok_y, kfw, bc2(0.0f));
    total = sel2(ok_x, ok_y, tot, bc2(0.0f));
}

constexpr int kFoldPairs = 16;


// Set slots of a multi-set launch (MULTI): see SetsLayout.
struct SetsArg {
    int per_cta, lanes, parent_tiles;
    size_t spline_stride;
    const SetTable* table;
};

// Shared-memory bytes of one set slot's spline tables: the T-typed log S coefficients, the
// pre-scaled FP32 rows with their edge rows (FP32 build) and the knots.
template <typename T>
__host__ __device__ inline size_t k2_slot_bytes(int n)
{
    const size_t b = sizeof(T) * 4 * (size_t)(n - 1) + (sizeof(T) == sizeof(float) ? sizeof(float4) * (size_t)(n + 1) : 0) +
                     sizeof(T) * (size_t)n;
    return (b + 15) & ~(size_t)15;
}

// MULTI = false: one parameter set, lanes = the CTA's threads.  MULTI = true: thread t holds
// set slot t / lanes of its group (its own spline tables in shared memory) and parent slot
// tile * lanes + t % lanes of that set's active list; a tile stages `lanes` samples per slot,
// each slot's records from its own set's amplitudes, while the Sobol points (one seed for all
// sets) and the geometry are the same for every slot.
template <typename T, bool SYM, int COUPLING, bool MULTI>
__global__ void __launch_bounds__(448, (sizeof(T) == 4 ? 2 : 1)) k2kf_kernel(Phys<T> ph, K2Box<T> box, SobolDirsArg dirs,
                                                    const double* __restrict__ r_grid, int n,
                                                    const double* __restrict__ spline,
                                                    const int32_t* __restrict__ active,
                                                    const int32_t* __restrict__ count, uint64_t offset,
                                                    uint64_t samples, double* __restrict__ partial, SetsArg sa)
{
    const int slots = MULTI ? sa.per_cta : 1;
    const int lanes = MULTI ? sa.lanes : (int)blockDim.x;
    const int my_slot = MULTI ? (int)threadIdx.x / lanes : 0;
    const int lt = (int)threadIdx.x - my_slot * lanes;
    const int group = MULTI ? (int)blockIdx.y / sa.parent_tiles : 0;
    const int ptile = MULTI ? (int)blockIdx.y - group * sa.parent_tiles : (int)blockIdx.y;
    int my_set = 0;
    uint64_t my_samples = samples, max_samples = samples;
    if (MULTI) {
        my_set = sa.table->slot_set[group * slots + my_slot];
        my_samples = my_set >= 0 ? sa.table->samples[my_set] : 0;
        // slot 0 of a group holds its largest budget
        max_samples = sa.table->samples[sa.table->slot_set[group * slots]];
    }
    const uint64_t tile = lanes;
    const uint64_t tiles = (max_samples + tile - 1) / tile;
    // MULTI: a CTA past its group's tiles has nothing to add (the finalize reads only the CTAs
    // below the tile count)
    if (MULTI && blockIdx.x >= tiles) return;

    extern __shared__ __align__(16) unsigned char k2_smem[];
    K2Rec<T>* recs = reinterpret_cast<K2Rec<T>*>(k2_smem);  // [blockDim.x], 16-byte aligned rows
    unsigned char* slot_base = reinterpret_cast<unsigned char*>(recs + blockDim.x);
    const size_t slot_bytes = k2_slot_bytes<T>(n);
    uint32_t* st = reinterpret_cast<uint32_t*>(slot_base + slots * slot_bytes);  // per slot [4][30] + shift[4]
    // slot q: cs [n-1][4] natural units, cs2 [n+1] pre-scaled with edge rows (FP32 path), xs [n]
    auto cs_of = [&](int q) { return reinterpret_cast<T*>(slot_base + q * slot_bytes); };
    auto cs2_of = [&](int q) { return reinterpret_cast<float4*>(cs_of(q) + 4 * (n - 1)); };
    auto xs_of = [&](int q) {
        return reinterpret_cast<T*>(cs2_of(q) + (sizeof(T) == sizeof(float) ? n + 1 : 0));
    };
    const double h64 = (spline[n - 1] - spline[0]) / (double)(n - 1);
    for (int q = 0; q < slots; ++q) {
        const int set_q = MULTI ? sa.table->slot_set[group * slots + q] : 0;
        if (set_q < 0) continue;
        const double* sp = spline + (MULTI ? (size_t)set_q * sa.spline_stride : 0);
        const double* src_coef = sp + n + 4 * (size_t)(n - 1);  // log S block
        T* cs = cs_of(q);
        float4* cs2 = cs2_of(q);
        T* xs = xs_of(q);
        for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = (T)sp[i];
        for (int i = threadIdx.x; i < 4 * (n - 1); i += blockDim.x) cs[i] = (T)src_coef[i];
        if (sizeof(T) == sizeof(float)) {
            const double l2e = 1.4426950408889634;
            for (int i = threadIdx.x; i < n - 1; i += blockDim.x) {
                const double* c = src_coef + 4 * (size_t)i;
                cs2[i + 1] = make_float4((float)(c[0] * l2e), (float)(c[1] * h64 * l2e),
                                         (float)(c[2] * h64 * h64 * l2e), (float)(c[3] * h64 * h64 * h64 * l2e));
            }
            if (threadIdx.x == 0) {
                cs2[0] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                cs2[n] = make_float4(-150.0f, 0.0f, 0.0f, 0.0f);
            }
        }
    }
    if (MULTI) {  // each slot's own Sobol directions
        for (int i = threadIdx.x; i < slots * kSetDirsWords; i += blockDim.x) {
            const int q = i / kSetDirsWords;
            const int set_q = sa.table->slot_set[group * slots + q];
            st[i] = set_q >= 0 ? sa.table->dirs[set_q][i - q * kSetDirsWords] : 0u;
        }
    } else {
        for (int i = threadIdx.x; i < 120; i += blockDim.x) st[i] = dirs.state[i / 30][i % 30];
        if (threadIdx.x < 4) st[120 + threadIdx.x] = dirs.shift[threadIdx.x];
    }
    __syncthreads();
    // this thread's slot (an empty slot reads slot 0's tables and prepares zero-weight records)
    const int view = MULTI && my_set < 0 ? 0 : my_slot;
    const uint32_t* my_st = st + (MULTI ? view * kSetDirsWords : 0);
    SplineView<T> s;
    s.x = xs_of(view);
    s.coef = cs_of(view);
    s.n = n;
    s.x0 = s.x[0];
    s.inv_h = (T)((double)(n - 1) / (spline[n - 1] - spline[0]));

    // per-evaluation spline: uniform-grid FP32 form in the mixed build, the exact
    // knot search in the FP64 build
    FastSpline fs;
    fs.coef = cs2_of(view);
    fs.u_scale = (float)(0.5 * 0.69314718055994531 / h64);
    fs.u_off = (float)(-spline[0] / h64);
    fs.u_top = (float)(n - 1);

    const int32_t* act = active + (MULTI && my_set > 0 ? (size_t)my_set * n : 0);
    const int n_active = MULTI ? (my_set >= 0 ? count[my_set] : 0) : *count;
    const int slot = ptile * lanes + lt;
    const bool has_parent = slot < n_active;
    K2Parent<T> P;
    K2ParentF PF;
    {
        const double r = has_parent ? r_grid[act[slot]] : 1.0;
        P.r = (T)r;
        P.r2 = P.r * P.r;
        P.lr = (T)log(r);
        P.two_r = (T)2 * P.r;
        PF.r = (float)r;
        PF.r2 = (float)(r * r);
        PF.lr = (float)log(r);
        PF.two_r = (float)(2.0 * r);
        PF.four_r = (float)(4.0 * r);
        P.alpha_r = alpha_of_log(P.lr, ph);
        PF.alpha_r = (float)P.alpha_r;
    }
    double acc_k2 = 0.0, acc_kf = 0.0, acc_sq = 0.0;
    // CTAs whose parent tile is empty still stage samples for nobody: skip them.
    const bool any_parent =
        MULTI ? __syncthreads_or(has_parent) != 0 : blockIdx.y * blockDim.x < (unsigned)n_active;
    if (any_parent) {
        // this slot's records start at record my_slot * lanes (pair my_slot * lanes / 2)
        const size_t rec0 = (size_t)my_slot * lanes;
        for (uint64_t tix = blockIdx.x; tix < tiles; tix += gridDim.x) {
            const uint64_t local = tix * tile + lt;
            const uint64_t done = tix * tile;
            const uint64_t remaining = my_samples > done ? my_samples - done : 0;
            const int count_here = (int)(remaining < tile ? remaining : tile);
            if constexpr (sizeof(T) == sizeof(float)) {
                // pair layout: the fields of samples 2p and 2p+1 side by side (lanes is even;
                // a padding sample past the budget carries zero weight)
                float rec[kRecLen];
                k2_prepare<float>(s, box, my_st, my_st + 120, offset + local, local < my_samples, rec);
                float* dst = reinterpret_cast<float*>(recs) + (size_t)(threadIdx.x >> 1) * (2 * kRecLen) +
                             (threadIdx.x & 1);
#pragma unroll
                for (int f = 0; f < kRecLen; ++f) dst[2 * f] = rec[f];
                __syncthreads();
                if (has_parent) {
                    const float4* pr = reinterpret_cast<const float4*>(recs) + (rec0 / 2) * (kRecLen / 2);
                    f2 sq = bc2(0.0f);  // variance estimate only: plain sum per tile
                    const int pairs = (count_here + 1) >> 1;
                    // FP32x2 partial sums of 16 pairs (32 samples), folded into FP64: the
                    // rounding of a 32-term FP32 sum instead of compensated summation.  The
                    // sums are of K2 + Kf and of Kf (K2 is their difference, formed once at
                    // the end): the total is needed anyway for the variance, and this saves
                    // the finite-test select of K2 per sample
                    for (int j0 = 0; j0 < pairs; j0 += kFoldPairs) {
                        const int jn = j0 + kFoldPairs < pairs ? j0 + kFoldPairs : pairs;
                        f2 ptot = bc2(0.0f), pkf = bc2(0.0f);
                        for (int j = j0; j < jn; ++j) {
                            f2 kfw, tot;
                            k2_pair_fast<SYM, COUPLING>(fs, ph, PF, pr + (kRecLen / 2) * j, kfw, tot);
                            ptot = add2(ptot, tot);
                            pkf = add2(pkf, kfw);
                            sq = fma2(tot, tot, sq);
                        }
                        acc_k2 += (double)ptot.x + (double)ptot.y;  // K2 + Kf until the end
                        acc_kf += (double)pkf.x + (double)pkf.y;
                    }
                    acc_sq += (double)sq.x + (double)sq.y;
                }
            } else {
                k2_prepare<T>(s, box, my_st, my_st + 120, offset + local, local < my_samples, recs[threadIdx.x].v);
                __syncthreads();
                if (has_parent) {
                    Kahan<T> sk2, skf;
                    sk2.reset();
                    skf.reset();
                    T sq = (T)0;  // variance estimate only: plain sum per tile
                    for (int j = 0; j < count_here; ++j) {
                        T k2w, kfw;
                        k2_point<T, SYM>(s, ph, P, recs[rec0 + j].v, k2w, kfw);
                        sk2.add(k2w);
                        skf.add(kfw);
                        const T tot = k2w + kfw;
                        sq += tot * tot;
                    }
                    acc_k2 += (double)sk2.sum - (double)sk2.comp;
                    acc_kf += (double)skf.sum - (double)skf.comp;
                    acc_sq += (double)sq;
                }
            }
            __syncthreads();
        }
    }
    double* o = nullptr;
    if (MULTI)
        o = partial + (((size_t)blockIdx.y * gridDim.x + blockIdx.x) * blockDim.x + threadIdx.x) * 3;
    else if (slot < n)
        o = partial + ((size_t)blockIdx.x * n + slot) * 3;
    if (o) {
        o[0] = sizeof(T) == sizeof(float) ? acc_k2 - acc_kf : acc_k2;
        o[1] = acc_kf;
        o[2] = acc_sq;
    }
}

// One warp per active parent: lanes add strided CTA partials, then a fixed
// shuffle tree combines them (the order does not depend on timing).
__global__ void __launch_bounds__(256) k2kf_finalize_kernel(const double* __restrict__ partial, int blocks, int n,
                                                            const int32_t* __restrict__ active,
                                                            const int32_t* __restrict__ count,
                                                            double* __restrict__ out)
{
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (slot >= n || slot >= *count) return;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int c = lane; c < blocks; c += 32) {
        const double* p = partial + ((size_t)c * n + slot) * 3;
        s0 += p[0];
        s1 += p[1];
        s2 += p[2];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
        double* o = out + 3 * (size_t)active[slot];
        o[0] = s0;
        o[1] = s1;
        o[2] = s2;
    }
}

// Multi-set finalize: one warp per (set blockIdx.y, active parent); the set's slot gives its
// CTA row and lane, and the CTAs below its group's tile count hold its partial sums.
__global__ void __launch_bounds__(256) k2kf_finalize_sets_kernel(const double* __restrict__ partial, int blocks,
                                                                 int threads, int n, SetsArg sa,
                                                                 const int32_t* __restrict__ active,
                                                                 const int32_t* __restrict__ count,
                                                                 double* __restrict__ out)
{
    const int slot = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int set = blockIdx.y;
    if (slot >= n || slot >= count[set]) return;
    const int set_slot = sa.table->set_slot[set];
    const int group = set_slot / sa.per_cta, q = set_slot - group * sa.per_cta;
    const int row = group * sa.parent_tiles + slot / sa.lanes;
    const int thread = q * sa.lanes + slot % sa.lanes;
    const uint64_t max_samples = sa.table->samples[sa.table->slot_set[group * sa.per_cta]];
    const uint64_t tiles = (max_samples + sa.lanes - 1) / sa.lanes;
    const int used = (uint64_t)blocks < tiles ? blocks : (int)tiles;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int c = lane; c < used; c += 32) {
        const double* p = partial + (((size_t)row * blocks + c) * threads + thread) * 3;
        s0 += p[0];
        s1 += p[1];
        s2 += p[2];
    }
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, o);
        s1 += __shfl_down_sync(0xffffffffu, s1, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
        double* o = out + 3 * ((size_t)set * n + active[(size_t)set * n + slot]);
        o[0] = s0;
        o[1] = s1;
        o[2] = s2;
    }
}

template <typename T>
K2Box<T> make_box(const nlo_bk_params& p, const nlo_bk_box& box, bool sym)
{
    K2Box<T> kb;
    double volume = 1.0;
    for (int d = 0; d < 4; ++d) {
        kb.lower[d] = (T)box.lower[d];
        kb.width[d] = (T)box.width[d];
    }
    if (sizeof(T) == sizeof(float)) {
        const float v01 = (float)box.width[0] * (float)box.width[1];
        const float v23 = (float)box.width[2] * (float)box.width[3];
        volume = (double)(v01 * v23);
    } else {
        volume = box.width[0] * box.width[1] * box.width[2] * box.width[3];
    }
    // the FP32 path folds the symmetrisation's 1/2 into the per-sample weight
    const double half = (sizeof(T) == sizeof(float) && sym) ? 0.5 : 1.0;
    kb.cpt_scale = (T)(half * volume * p.nc * p.nc / (8.0 * kPi * kPi * kPi * kPi));
    return kb;
}

template <typename T>
size_t k2_smem_bytes(int threads, int slots, int points)
{
    return sizeof(K2Rec<T>) * threads + slots * k2_slot_bytes<T>(points) + sizeof(uint32_t) * kSetDirsWords * slots;
}

template <typename T, bool SYM, int COUPLING>
cudaError_t launch_sets_typed(const nlo_bk_params& p, const double* r, int points, const double* spline,
                              size_t spline_stride, const int32_t* active, const int32_t* counts,
                              const nlo_bk_box& box, const SetsLayout& L, const SetTable* table, double* partial,
                              cudaStream_t stream)
{
    const size_t smem = k2_smem_bytes<T>(L.threads, L.per_cta, points);
    cudaError_t e = raise_dynamic_smem((const void*)k2kf_kernel<T, SYM, COUPLING, true>, smem);
    if (e == cudaSuccess) e = prefer_shared_carveout((const void*)k2kf_kernel<T, SYM, COUPLING, true>);
    if (e != cudaSuccess) return e;
    SetsArg sa{L.per_cta, L.lanes, L.parent_tiles, spline_stride, table};
    dim3 grid((unsigned)L.blocks, (unsigned)(L.groups * L.parent_tiles));
    SobolDirsArg unused;
    std::memset(&unused, 0, sizeof(unused));
    k2kf_kernel<T, SYM, COUPLING, true><<<grid, L.threads, smem, stream>>>(
        make_phys<T>(p), make_box<T>(p, box, SYM), unused, r, points, spline, active, counts, 0, 0, partial, sa);
    return cudaGetLastError();
}

template <typename T, bool SYM, int COUPLING>
cudaError_t launch_typed(const nlo_bk_params& p, const double* r, int points, const double* spline,
                         const int32_t* active, const int32_t* count, const SobolDirsArg& dirs, uint64_t offset,
                         uint64_t samples, const nlo_bk_box& box, double* partial, int max_blocks, int threads,
                         int parent_tiles, int* used_blocks, cudaStream_t stream)
{
    const size_t smem = k2_smem_bytes<T>(threads, 1, points);
    cudaError_t e = raise_dynamic_smem((const void*)k2kf_kernel<T, SYM, COUPLING, false>, smem);
    if (e == cudaSuccess) e = prefer_shared_carveout((const void*)k2kf_kernel<T, SYM, COUPLING, false>);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2kf_kernel<T, SYM, COUPLING, false>, threads, smem);
    if (e != cudaSuccess) return e;
    int device = 0, sms = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (per_sm < 1) per_sm = 1;
    const uint64_t tiles = (samples + threads - 1) / threads;
    uint64_t blocks = (uint64_t)per_sm * sms / (uint64_t)parent_tiles;
    if (blocks < 1) blocks = 1;
    if (blocks > (uint64_t)max_blocks) blocks = (uint64_t)max_blocks;
    if (blocks > tiles) blocks = tiles;
    *used_blocks = (int)blocks;
    dim3 grid((unsigned)blocks, (unsigned)parent_tiles);
    k2kf_kernel<T, SYM, COUPLING, false><<<grid, threads, smem, stream>>>(
        make_phys<T>(p), make_box<T>(p, box, SYM), dirs, r, points, spline, active, count, offset, samples, partial,
        SetsArg{});
    return cudaGetLastError();
}

// The kernel instantiation of a parameter set: FP64 (one form for every coupling) or the
// FP32 coupling variant; f(T(), SYM, COUPLING) with std::integral_constant tags.
template <class F>
cudaError_t dispatch_variant(const nlo_bk_params& p, F f)
{
    using std::integral_constant;
    const bool sym = p.symmetrize != 0;
    const int coupling = p.fixed_coupling                 ? 2
                         : p.rc_nlo == NLO_RC_NLO_PARENT ? 4
                         : p.nf > 3.0                    ? 3
                         : p.alpha_cap > 0.0             ? 1
                                                         : 0;
#define NLO_K2_VARIANT(T, C)                                                                  \
    (sym ? f(T(), integral_constant<bool, true>(), integral_constant<int, C>())                \
         : f(T(), integral_constant<bool, false>(), integral_constant<int, C>()))
    if (p.precision == NLO_PRECISION_FP64) return NLO_K2_VARIANT(double, 0);
    switch (coupling) {
        case 0: return NLO_K2_VARIANT(float, 0);
        case 1: return NLO_K2_VARIANT(float, 1);
        case 2: return NLO_K2_VARIANT(float, 2);
        case 3: return NLO_K2_VARIANT(float, 3);
        default: return NLO_K2_VARIANT(float, 4);
    }
#undef NLO_K2_VARIANT
}

// at most 448 lanes (parents) per CTA: the FP32 kernel's bounds (448 threads, two CTAs per
// SM) give it 72 registers without spills; larger grids take several parent tiles
constexpr int kLaneCap = 448;

}  // namespace

cudaError_t launch_k2kf(const nlo_bk_params& p, const double* r, int points, const double* spline,
                        const int32_t* active, const int32_t* count, const SobolDirsArg& dirs, uint64_t offset,
                        uint64_t samples, const nlo_bk_box& box, double* out, double* partial, int max_blocks,
                        cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * 3 * (size_t)points, stream);
    if (e != cudaSuccess || samples == 0) return e;
    int threads = ((points < kLaneCap ? points : kLaneCap) + 31) / 32 * 32;
    if (threads < 64) threads = 64;
    const int parent_tiles = (points + threads - 1) / threads;
    int used = 0;
    e = dispatch_variant(p, [&](auto t, auto sym, auto c) {
        return launch_typed<decltype(t), decltype(sym)::value, decltype(c)::value>(
            p, r, points, spline, active, count, dirs, offset, samples, box, partial, max_blocks, threads, parent_tiles,
            &used, stream);
    });
    if (e != cudaSuccess) return e;
    k2kf_finalize_kernel<<<(points * 32 + 255) / 256, 256, 0, stream>>>(partial, used, points, active, count, out);
    return cudaGetLastError();
}

SetsLayout sets_layout(int points, int sets, int waves)
{
    SetsLayout L;
    L.lanes = ((points < kLaneCap ? points : kLaneCap) + 31) / 32 * 32;
    if (L.lanes < 64) L.lanes = 64;
    L.per_cta = kLaneCap / L.lanes;
    if (L.per_cta > sets) L.per_cta = sets;
    if (L.per_cta < 1) L.per_cta = 1;
    L.parent_tiles = (points + L.lanes - 1) / L.lanes;
    L.groups = (sets + L.per_cta - 1) / L.per_cta;
    L.threads = L.per_cta * L.lanes;
    int device = 0, sms = 148;
    if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (sms < 1) sms = 148;
    // about `waves` waves of the FP32 kernel's two CTAs per SM over all groups and parent
    // tiles; a group with fewer tiles than CTAs leaves the rest idle (they return at once)
    const long rows = (long)L.groups * L.parent_tiles;
    long blocks = ((long)(waves < 1 ? 1 : waves) * 2 * sms + rows - 1) / rows;
    if (blocks > 4L * sms) blocks = 4L * sms;
    L.blocks = (int)(blocks < 1 ? 1 : blocks);
    return L;
}

cudaError_t launch_k2kf_sets(const nlo_bk_params& p, const double* r, int points, int sets, const double* spline,
                             size_t spline_stride, const int32_t* active, const int32_t* counts,
                             const nlo_bk_box& box, const SetsLayout& L, const SetTable* table, double* out,
                             double* partial, cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * 3 * (size_t)points * sets, stream);
    if (e != cudaSuccess) return e;
    e = dispatch_variant(p, [&](auto t, auto sym, auto c) {
        return launch_sets_typed<decltype(t), decltype(sym)::value, decltype(c)::value>(
            p, r, points, spline, spline_stride, active, counts, box, L, table, partial, stream);
    });
    if (e != cudaSuccess) return e;
    SetsArg sa{L.per_cta, L.lanes, L.parent_tiles, spline_stride, table};
    k2kf_finalize_sets_kernel<<<dim3((points * 32 + 255) / 256, sets), 256, 0, stream>>>(
        partial, L.blocks, L.threads, points, sa, active, counts, out);
    return cudaGetLastError();
}

}  // namespace nlo
