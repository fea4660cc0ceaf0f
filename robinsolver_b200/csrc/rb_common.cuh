// rb_common.cuh -- complex FP64 helpers and the strided/gathered matrix views shared by
// every kernel of the B200 HPS factor/solve.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <climits>
#include <cstdint>

namespace rb {

using z = double2;  // interleaved complex128: x = re, y = im

__host__ __device__ __forceinline__ z zmk(double re, double im) { return make_double2(re, im); }
__host__ __device__ __forceinline__ z zadd(z a, z b) { return zmk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ z zsub(z a, z b) { return zmk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ z zneg(z a) { return zmk(-a.x, -a.y); }
__host__ __device__ __forceinline__ z zmul(z a, z b) {
    return zmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ z zscale(double s, z a) { return zmk(s * a.x, s * a.y); }
// acc += a*b with four FMAs
__device__ __forceinline__ void zfma(z& acc, z a, z b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
// acc -= a*b
__device__ __forceinline__ void zfms(z& acc, z a, z b) {
    acc.x = fma(-a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(-a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
}
// 1/a = (re - i im) / (re^2 + im^2), with one division: a pivot's reciprocal sits on the
// Gauss-Jordan critical path, where a second division costs ~20% of the pivot step
__host__ __device__ __forceinline__ z zrcp(z a) {
    const double r = 1.0 / (a.x * a.x + a.y * a.y);
    return zmk(a.x * r, -a.y * r);
}
// |re| + |im|: the magnitude LAPACK's izamax ranks pivots by
__host__ __device__ __forceinline__ double zabs1(z a) { return fabs(a.x) + fabs(a.y); }

// A matrix view: logical element (i, j) lives at p[row(i) + col(j) * ld], where row(i) is
// rmap[i] when a map is given, else i shifted past a skipped band [rs, rs + rl) (same for
// columns).  Maps and bands express the face gathers of the merge (non-interface faces of
// a child) without copies.
struct ZView {
    const z* p;
    const int* rmap;
    const int* cmap;
    long long ld;
    int rs, rl, cs, cl;
};
struct ZOut {
    z* p;
    const int* rmap;
    const int* cmap;
    long long ld;
    int rs, rl, cs, cl;
};

__host__ __device__ __forceinline__ ZView zview(const z* p, long long ld) {
    ZView v;
    v.p = p; v.rmap = nullptr; v.cmap = nullptr; v.ld = ld;
    v.rs = INT_MAX; v.rl = 0; v.cs = INT_MAX; v.cl = 0;
    return v;
}
__host__ __device__ __forceinline__ ZOut zout(z* p, long long ld) {
    ZOut v;
    v.p = p; v.rmap = nullptr; v.cmap = nullptr; v.ld = ld;
    v.rs = INT_MAX; v.rl = 0; v.cs = INT_MAX; v.cl = 0;
    return v;
}
template <class V>
__device__ __forceinline__ int vrow(const V& v, int i) {
    return v.rmap ? __ldg(v.rmap + i) : (i + (i >= v.rs ? v.rl : 0));
}
template <class V>
__device__ __forceinline__ int vcol(const V& v, int j) {
    return v.cmap ? __ldg(v.cmap + j) : (j + (j >= v.cs ? v.cl : 0));
}

// One complex GEMM problem: D(i,j) = alpha * sum_k A(i,k) B(k,j) + beta * C(i,j)
// (the beta term only when C.p != nullptr, and not for rows in [nobeta_r0, nobeta_r1);
// C may alias D).
struct GemmDesc {
    ZView A, B, C;
    ZOut D;
    z alpha, beta;
    int m, n, k;
    int nobeta_r0, nobeta_r1;
    int pad;
};

// A batch of GEMM problems resident in device memory, with the largest sizes for grid setup.
struct GemmBatch {
    GemmDesc* d_desc = nullptr;
    int count = 0;
    int max_m = 0, max_n = 0, max_k = 0;
    double flops = 0.0;   // 8*m*n*k summed
    // DFMA kernels only: every DFMA tile shape accumulates an element's k-sum in the same order,
    // so results do not depend on the batch's sizes (used for the solve, whose n = RHS count)
    bool fixed_order = false;
    // split-K (fixed-order batches only): k is cut into ksplit ranges of kchunk, whose raw sums
    // go to work (pstride elements per range and problem, ld max_m) and are then added in range
    // order.  ksplit depends on count, m and k only, never on n.
    int ksplit = 1;
    int kchunk = 0;
    z* work = nullptr;
    long long pstride = 0;
    // every problem's k runs contiguously through both operands (gemm_k_contiguous), so operand
    // copies may advance by a fixed stride per k-tile
    bool kcontig = false;
    // split-K of the same batch on the tcgen05 kernel (128-row tiles): t5_ksplit ranges of
    // t5_kchunk, raw sums in `work` (t5_pstride elements per range and problem, ld max_m)
    int t5_ksplit = 1;
    int t5_kchunk = 0;
    long long t5_pstride = 0;
    // the tcgen05 kernel's operand planes (tc5_plane_bytes(batch) bytes, 256-byte aligned): every
    // operand element split once into four TF32 parts and laid out block by block as the kernel's
    // shared-memory stages hold them
    void* t5_planes = nullptr;
    size_t t5_plane_cap = 0;      // bytes at t5_planes; a launch that needs more is refused
    // arithmetic of the tensor-core engine: 0 split TF32 ("TF32x3"), 1 int8 digit slices with
    // exact integer accumulation (Ozaki scheme); -1: the process default (tc5_engine)
    int t5_engine = -1;
    // FP64 engine (tile shape) chosen by an autotuner; -1: the launcher's own rule
    int engine = -1;
};

// A(i, k) sits at A.p[row(i) + k * A.ld] and B(k, j) at B.p[k + col(j) * B.ld] for every k < K:
// no map on A's columns or B's rows, and no skipped band that starts below K
__host__ __device__ inline bool gemm_k_contiguous(const GemmDesc& g) {
    return !g.A.cmap && (g.A.cl == 0 || g.A.cs >= g.k) && !g.B.rmap && (g.B.rl == 0 || g.B.rs >= g.k);
}

}  // namespace rb
