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
// values, the kernels and the coupling remain.  Lane sums are compensated FP32
// (Kahan) per tile, folded into FP64 per lane; per-CTA partials go to the caller's
// workspace and a second kernel adds them in a fixed order (deterministic).

#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "sobol.cuh"

namespace nlo {

namespace {

// Per-sample record (r-independent), 20 values.
enum Rec {
    kZ, kZ2, kS1, kS2, kP1, kP2, kU1, kV1, kU2, kV2,
    kQ, kD1, kD2, kDN, kSY, kLmin, kCpt, kDl, kZsq, kZ2sq,
    kRecLen
};

template <typename T>
struct alignas(16) K2Rec {
    T v[kRecLen];
};

template <typename T>
struct K2Box {
    T lower[4], width[4];
    T cpt_scale;  // volume * Nc^2 / (8 pi^4)
};

// atanh(t)/t - 1 = t^2 sum_{k>=1} t^{2k-2}/(2k+1); 14 terms reach FP32 (and, with
// |t| < 0.5, ~1e-9 relative in FP64 -- the FP64 build uses more terms).
template <typename T>
__device__ __forceinline__ T atanh_ratio_m1(T t2);

template <>
__device__ __forceinline__ float atanh_ratio_m1<float>(float t2)
{
    float s = 1.0f / 29.0f;
    s = fmaf(s, t2, 1.0f / 27.0f);
    s = fmaf(s, t2, 1.0f / 25.0f);
    s = fmaf(s, t2, 1.0f / 23.0f);
    s = fmaf(s, t2, 1.0f / 21.0f);
    s = fmaf(s, t2, 1.0f / 19.0f);
    s = fmaf(s, t2, 1.0f / 17.0f);
    s = fmaf(s, t2, 1.0f / 15.0f);
    s = fmaf(s, t2, 1.0f / 13.0f);
    s = fmaf(s, t2, 1.0f / 11.0f);
    s = fmaf(s, t2, 1.0f / 9.0f);
    s = fmaf(s, t2, 1.0f / 7.0f);
    s = fmaf(s, t2, 1.0f / 5.0f);
    s = fmaf(s, t2, 1.0f / 3.0f);
    return s * t2;
}

template <>
__device__ __forceinline__ double atanh_ratio_m1<double>(double t2)
{
    double s = 0.0;
#pragma unroll
    for (int k = 30; k >= 1; --k) s = fma(s, t2, 1.0 / (2.0 * k + 1.0));
    return s * t2;
}

template <typename T>
__device__ __forceinline__ void k2_prepare(const SplineView<T>& s, const Phys<T>& ph, const K2Box<T>& box,
                                           const uint32_t* state, const uint32_t* shift, uint64_t index, bool valid,
                                           T* rec)
{
    T u[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) u[d] = sobol_unit<T>(sobol_bits(state + 30 * d, shift[d], index), index);
    T x[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) x[d] = M<T>::add_rn(box.lower[d], M<T>::mul_rn(box.width[d], u[d]));
    const T lz = x[0], lz2 = x[1], th = x[2], th2 = x[3];
    const T z = M<T>::exp_acc(lz), z2 = M<T>::exp_acc(lz2);
    const T sh1 = M<T>::sin((T)0.5 * th), sh2 = M<T>::sin((T)0.5 * th2);
    const T c1 = M<T>::cos(th), c2 = M<T>::cos(th2);
    const T dth = th - th2;
    const T c12 = M<T>::cos(dth), sh12 = M<T>::sin((T)0.5 * dth);
    const T zzsq = (z - z2) * (z - z2) + (T)4 * z * z2 * sh12 * sh12;
    valid = valid && zzsq >= M<T>::tiny_square();
    const T lzz = (T)0.5 * M<T>::log_acc(zzsq);
    const NS<T> Y = eval_s_log(s, lz), Y2 = eval_s_log(s, lz2), ZZ = eval_s_log(s, lzz);
    const T dN = ndiff_s(Y2, Y);  // N_Y2 - N_Y
    rec[kZ] = z;
    rec[kZ2] = z2;
    rec[kS1] = sh1 * sh1;
    rec[kS2] = sh2 * sh2;
    rec[kP1] = (z2 - z) * (z2 + z);
    rec[kP2] = (T)2 * z * z2 * (z2 * c1 - z * c2);
    rec[kU1] = z2 - z * c12;
    rec[kV1] = z * (z * c2 - z2 * c1);
    rec[kU2] = z - z2 * c12;
    rec[kV2] = z2 * (z2 * c1 - z * c2);
    rec[kQ] = valid ? M<T>::rcp(zzsq) : (T)0;
    // S_Y - S_zz S_Y2 = S_Y N_zz + S_zz (N_Y2 - N_Y);  S_Y2 - S_zz S_Y = S_Y2 N_zz - S_zz (N_Y2 - N_Y)
    rec[kD1] = Y.S * ZZ.N + ZZ.S * dN;
    rec[kD2] = Y2.S * ZZ.N - ZZ.S * dN;
    rec[kDN] = dN;
    rec[kSY] = Y.S;
    rec[kLmin] = M<T>::fmin(M<T>::fmin(lz, lz2), lzz);
    rec[kCpt] = valid ? box.cpt_scale * M<T>::exp_acc((T)2 * lz + (T)2 * lz2) : (T)0;
    rec[kDl] = (T)2 * (lz2 - lz);
    rec[kZsq] = z * z;
    rec[kZ2sq] = z2 * z2;
}

template <typename T>
struct K2Parent {
    T r, r2, lr, two_r;
};

// K2 and Kf contributions of one sample to one parent (already weighted).
template <typename T, bool SYM>
__device__ __forceinline__ void k2_point(const SplineView<T>& s, const Phys<T>& ph, const K2Parent<T>& P,
                                         const T* __restrict__ rec, T& k2w, T& kfw)
{
    const T r = P.r;
    const T z = rec[kZ], z2 = rec[kZ2];
    const T Xsq = (r - z) * (r - z) + (T)4 * r * z * rec[kS1];
    const T X2sq = (r - z2) * (r - z2) + (T)4 * r * z2 * rec[kS2];
    const bool valid = Xsq >= M<T>::tiny_square() && X2sq >= M<T>::tiny_square();
    const T lXs = M<T>::log_fast(Xsq), lX2s = M<T>::log_fast(X2sq);
    const NS<T> vX = eval_s_log(s, (T)0.5 * lXs), vX2 = eval_s_log(s, (T)0.5 * lX2s);
    // kernels (k2.py, kf.py) in the stable form
    const T a = Xsq * rec[kZ2sq], b = X2sq * rec[kZsq];
    const T sab = a + b;
    const T rs = M<T>::rcp(sab);
    const T d = r * (r * rec[kP1] - rec[kP2]);
    const T t = d * rs;
    const T t2 = t * t;
    T hm1, Ld;
    if (t2 < (T)0.25) {
        hm1 = atanh_ratio_m1<T>(t2);
        Ld = (T)2 * t * ((T)1 + hm1);
    } else {
        Ld = lXs - lX2s + rec[kDl];  // log(a/b)
        hm1 = M<T>::div(Ld, (T)2 * t) - (T)1;
    }
    const T q = rec[kQ];
    const T L = (T)2 * ((T)1 + hm1) * rs;
    const T f = (T)2 * hm1;
    const T fq2 = f * q * q;
    const T r2Lq = P.r2 * L * q;
    const T C0 = fq2 - (T)4 * r2Lq;
    // L r^4/a + log(a/b) r^2 q/a = L r^2 q 2 r B1/(X^2 z'), B1 = r (z' - z c12) + z (z c2 - z' c1)
    const T B1 = r * rec[kU1] + rec[kV1];
    const T B2 = r * rec[kU2] + rec[kV2];
    T k2 = C0 + r2Lq * P.two_r * B1 * M<T>::rcp(Xsq * z2);
    T k2s = C0 + r2Lq * P.two_r * B2 * M<T>::rcp(X2sq * z);
    const T kf = (r2Lq - fq2) * ph.nf_over_nc;
    T dip = vX.S * rec[kD1];
    T dips = vX2.S * rec[kD2];
    if (M<T>::fabs(k2) > (T)1e10 && M<T>::fabs(dip) < (T)1e-10) { k2 = (T)0; dip = (T)0; }
    if (M<T>::fabs(k2s) > (T)1e10 && M<T>::fabs(dips) < (T)1e-10) { k2s = (T)0; dips = (T)0; }
    const T dNX = ndiff_s(vX, vX2);
    T k2part, fermion;
    if (SYM) {
        k2part = (T)0.5 * (k2 * dip + k2s * dips);
        fermion = (T)0.5 * kf * dNX * rec[kDN];
    } else {
        k2part = k2 * dip;
        fermion = kf * rec[kSY] * dNX;
    }
    if (!(ph.nf > (T)0)) fermion = (T)0;
    const T lmin = M<T>::fmin(M<T>::fmin(rec[kLmin], P.lr), (T)0.5 * M<T>::fmin(lXs, lX2s));
    const T alpha = alpha_of_log(lmin, ph);
    const T scale = alpha * alpha * rec[kCpt];
    k2w = k2part * scale;
    kfw = -fermion * scale;
    if (!valid || !M<T>::finite(k2w)) k2w = (T)0;
    if (!valid || !M<T>::finite(kfw)) kfw = (T)0;
}

template <typename T, bool SYM>
__global__ void __launch_bounds__(1024) k2kf_kernel(Phys<T> ph, K2Box<T> box, SobolDirsArg dirs,
                                                    const double* __restrict__ r_grid, int n,
                                                    const double* __restrict__ spline,
                                                    const int32_t* __restrict__ active,
                                                    const int32_t* __restrict__ count, uint64_t offset,
                                                    uint64_t samples, double* __restrict__ partial)
{
    extern __shared__ __align__(16) unsigned char k2_smem[];
    K2Rec<T>* recs = reinterpret_cast<K2Rec<T>*>(k2_smem);  // [blockDim.x]
    T* xs = reinterpret_cast<T*>(recs + blockDim.x);
    T* cs = xs + n;
    uint32_t* st = reinterpret_cast<uint32_t*>(cs + 4 * (n - 1));  // [4][30] + shift[4]
    const double* src_coef = spline + n + 4 * (size_t)(n - 1);     // log S block
    for (int i = threadIdx.x; i < n; i += blockDim.x) xs[i] = (T)spline[i];
    for (int i = threadIdx.x; i < 4 * (n - 1); i += blockDim.x) cs[i] = (T)src_coef[i];
    for (int i = threadIdx.x; i < 120; i += blockDim.x) st[i] = dirs.state[i / 30][i % 30];
    if (threadIdx.x < 4) st[120 + threadIdx.x] = dirs.shift[threadIdx.x];
    __syncthreads();
    SplineView<T> s;
    s.x = xs;
    s.coef = cs;
    s.n = n;
    s.x0 = xs[0];
    s.inv_h = (T)((double)(n - 1) / (spline[n - 1] - spline[0]));

    const int n_active = *count;
    const int slot = blockIdx.y * blockDim.x + threadIdx.x;
    const bool has_parent = slot < n_active;
    K2Parent<T> P;
    {
        const double r = has_parent ? r_grid[active[slot]] : 1.0;
        P.r = (T)r;
        P.r2 = P.r * P.r;
        P.lr = (T)log(r);
        P.two_r = (T)2 * P.r;
    }
    double acc_k2 = 0.0, acc_kf = 0.0, acc_sq = 0.0;
    const uint64_t tile = blockDim.x;
    const uint64_t tiles = (samples + tile - 1) / tile;
    // CTAs whose parent tile is empty still stage samples for nobody: skip them.
    const bool any_parent = blockIdx.y * blockDim.x < (unsigned)n_active;
    if (any_parent) {
        for (uint64_t tix = blockIdx.x; tix < tiles; tix += gridDim.x) {
            const uint64_t local = tix * tile + threadIdx.x;
            k2_prepare<T>(s, ph, box, st, st + 120, offset + local, local < samples, recs[threadIdx.x].v);
            __syncthreads();
            if (has_parent) {
                const uint64_t remaining = samples - tix * tile;
                const int count_here = (int)(remaining < tile ? remaining : tile);
                Kahan<T> sk2, skf;
                sk2.reset();
                skf.reset();
                for (int j = 0; j < count_here; ++j) {
                    T k2w, kfw;
                    k2_point<T, SYM>(s, ph, P, recs[j].v, k2w, kfw);
                    sk2.add(k2w);
                    skf.add(kfw);
                    const double tot = (double)k2w + (double)kfw;
                    acc_sq = fma(tot, tot, acc_sq);
                }
                acc_k2 += (double)sk2.sum - (double)sk2.comp;
                acc_kf += (double)skf.sum - (double)skf.comp;
            }
            __syncthreads();
        }
    }
    if (slot < n) {
        double* o = partial + ((size_t)blockIdx.x * n + slot) * 3;
        o[0] = acc_k2;
        o[1] = acc_kf;
        o[2] = acc_sq;
    }
}

__global__ void k2kf_finalize_kernel(const double* __restrict__ partial, int blocks, int n,
                                     const int32_t* __restrict__ active, const int32_t* __restrict__ count,
                                     double* __restrict__ out)
{
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= *count || slot >= n) return;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int c = 0; c < blocks; ++c) {
        const double* p = partial + ((size_t)c * n + slot) * 3;
        s0 += p[0];
        s1 += p[1];
        s2 += p[2];
    }
    double* o = out + 3 * (size_t)active[slot];
    o[0] = s0;
    o[1] = s1;
    o[2] = s2;
}

template <typename T, bool SYM>
cudaError_t launch_typed(const nlo_bk_params& p, const double* r, int points, const double* spline,
                         const int32_t* active, const int32_t* count, const SobolDirsArg& dirs, uint64_t offset,
                         uint64_t samples, const nlo_bk_box& box, double* partial, int max_blocks, int threads,
                         int parent_tiles, int* used_blocks, cudaStream_t stream)
{
    const size_t smem = sizeof(K2Rec<T>) * threads + sizeof(T) * (size_t)(points + 4 * (points - 1)) +
                        sizeof(uint32_t) * 124;
    cudaError_t e = cudaFuncSetAttribute(k2kf_kernel<T, SYM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k2kf_kernel<T, SYM>, threads, smem);
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
    kb.cpt_scale = (T)(volume * p.nc * p.nc / (8.0 * kPi * kPi * kPi * kPi));
    dim3 grid((unsigned)blocks, (unsigned)parent_tiles);
    k2kf_kernel<T, SYM><<<grid, threads, smem, stream>>>(make_phys<T>(p), kb, dirs, r, points, spline, active, count,
                                                        offset, samples, partial);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_k2kf(const nlo_bk_params& p, const double* r, int points, const double* spline,
                        const int32_t* active, const int32_t* count, const SobolDirsArg& dirs, uint64_t offset,
                        uint64_t samples, const nlo_bk_box& box, double* out, double* partial, int max_blocks,
                        cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * 3 * (size_t)points, stream);
    if (e != cudaSuccess || samples == 0) return e;
    const int cap = 1024;
    int threads = ((points < cap ? points : cap) + 31) / 32 * 32;
    if (threads < 64) threads = 64;
    const int parent_tiles = (points + threads - 1) / threads;
    int used = 0;
    const bool fp64 = p.precision == NLO_PRECISION_FP64;
    const bool sym = p.symmetrize != 0;
    if (fp64 && sym)
        e = launch_typed<double, true>(p, r, points, spline, active, count, dirs, offset, samples, box, partial,
                                       max_blocks, threads, parent_tiles, &used, stream);
    else if (fp64)
        e = launch_typed<double, false>(p, r, points, spline, active, count, dirs, offset, samples, box, partial,
                                        max_blocks, threads, parent_tiles, &used, stream);
    else if (sym)
        e = launch_typed<float, true>(p, r, points, spline, active, count, dirs, offset, samples, box, partial,
                                      max_blocks, threads, parent_tiles, &used, stream);
    else
        e = launch_typed<float, false>(p, r, points, spline, active, count, dirs, offset, samples, box, partial,
                                       max_blocks, threads, parent_tiles, &used, stream);
    if (e != cudaSuccess) return e;
    k2kf_finalize_kernel<<<(points + 127) / 128, 128, 0, stream>>>(partial, used, points, active, count, out);
    return cudaGetLastError();
}

}  // namespace nlo
