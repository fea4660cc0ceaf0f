// rb_gemm.cu -- descriptor-driven batched complex128 GEMM for sm_100a.
//
// One launch runs a whole batch of independent problems (all nodes of a tree level, all
// leaves of a tree): blockIdx.y picks the problem descriptor, blockIdx.x a C tile.  Operands
// are ZViews, so the merge's face gathers (non-interface rows/columns of a child's
// Robin-to-Robin matrix) and the scatter into the parent's face order happen inside the loads
// and the epilogue instead of in copy kernels.
//
// FP64 has no tcgen05 kind: the large problems run on the FP64 tensor-core MMA
// (mma.sync m8n8k4 .f64, rb_gemm_dmma.cuh), the small ones and the solve on DFMA register tiles
// (rb_gemm_tile.cuh).
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "rb_gemm_dmma.cuh"
#include "rb_gemm_tile.cuh"
#include "rb_kernels.h"

namespace rb {

template <int BM, int BN, int TM, int TN, int BK, int STAGES, int MINB>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), MINB)
zgemm_desc_kernel(const GemmDesc* __restrict__ descs) {
    constexpr int NT = (BM / TM) * (BN / TN);
    extern __shared__ z dfma_smem[];
    __shared__ GemmDesc sd;
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(descs + blockIdx.y);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
        for (int w = threadIdx.x; w < (int)(sizeof(GemmDesc) / 8); w += NT) dst[w] = src[w];
    }
    __syncthreads();
    zgemm_tile<BM, BN, TM, TN, BK, STAGES>(sd, blockIdx.x, dfma_smem);
}

// split-K pass: blockIdx.z picks the k range; raw sums go to the batch's workspace
template <int BM, int BN, int TM, int TN, int BK, int STAGES, int MINB>
__global__ void __launch_bounds__((BM / TM) * (BN / TN), MINB)
zgemm_split_kernel(const GemmDesc* __restrict__ descs, int kchunk, z* work, long long pstride, int ldp, int ksplit) {
    constexpr int NT = (BM / TM) * (BN / TN);
    extern __shared__ z dfma_smem[];
    __shared__ GemmDesc sd;
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(descs + blockIdx.y);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
        for (int w = threadIdx.x; w < (int)(sizeof(GemmDesc) / 8); w += NT) dst[w] = src[w];
    }
    __syncthreads();
    const int kb = blockIdx.z * kchunk;
    z* part = work + ((long long)blockIdx.y * ksplit + blockIdx.z) * pstride;
    zgemm_tile<BM, BN, TM, TN, BK, STAGES, true>(sd, blockIdx.x, dfma_smem, kb, kb + kchunk, part, ldp);
}

// split-K reduction: the ranges' sums added in range order, then the usual epilogue
__global__ void __launch_bounds__(256) zgemm_reduce_kernel(const GemmDesc* __restrict__ descs, const z* __restrict__ work,
                                                          long long pstride, int ldp, int ksplit) {
    const GemmDesc& g = descs[blockIdx.y];
    const int m = g.m, n = g.n;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)m * n) return;
    const int i = (int)(e % m), j = (int)(e / m);
    const z* p = work + (long long)blockIdx.y * ksplit * pstride + i + (long long)j * ldp;
    z acc = p[0];
    for (int r = 1; r < ksplit; ++r) acc = zadd(acc, p[r * pstride]);
    z v = zmul(g.alpha, acc);
    if (g.C.p && !(i >= g.nobeta_r0 && i < g.nobeta_r1)) zfma(v, g.beta, g.C.p[vrow(g.C, i) + (long long)vcol(g.C, j) * g.C.ld]);
    g.D.p[vrow(g.D, i) + (long long)vcol(g.D, j) * g.D.ld] = v;
}

template <int BM, int BN, int WM, int WN, int MINB>
__global__ void __launch_bounds__(32 * WM * WN, MINB) zgemm_dmma_kernel(const GemmDesc* __restrict__ descs) {
    extern __shared__ z dmma_smem[];
    __shared__ GemmDesc sd;
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(descs + blockIdx.y);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
        for (int w = threadIdx.x; w < (int)(sizeof(GemmDesc) / 8); w += 32 * WM * WN) dst[w] = src[w];
    }
    __syncthreads();
    zgemm_tile_dmma<BM, BN, WM, WN>(sd, blockIdx.x, dmma_smem);
}

// MINB CTAs per SM: the carveout is set to the largest shared-memory share so that they fit
template <int BM, int BN, int WM, int WN, int MINB>
static cudaError_t launch_dmma(const GemmBatch& b, cudaStream_t s) {
    using Cfg = DmmaCfg<BM, BN, WM, WN>;
    static DeviceAttrCache attr;
    {
        cudaError_t e = ensure_smem_attr(zgemm_dmma_kernel<BM, BN, WM, WN, MINB>, Cfg::SMEM_BYTES, attr, true);
        if (e != cudaSuccess) return e;
    }
    const int tiles = ((b.max_m + BM - 1) / BM) * ((b.max_n + BN - 1) / BN);
    for (int off = 0; off < b.count; off += 65535) {
        const int cnt = (b.count - off) < 65535 ? (b.count - off) : 65535;
        dim3 grid(tiles, cnt);
        zgemm_dmma_kernel<BM, BN, WM, WN, MINB><<<grid, Cfg::NT, Cfg::SMEM_BYTES, s>>>(b.d_desc + off);
        note_launch();
    }
    return cudaGetLastError();
}

// A view of the same matrix whose column j is column j + kb of v (B: row j is row j + kb)
__device__ __forceinline__ ZView view_from_col(ZView v, int kb) {
    if (v.cmap) {
        v.cmap += kb;
    } else if (v.cs >= kb) {
        v.p += (long long)kb * v.ld;
        if (v.cs != INT_MAX) v.cs -= kb;
    } else {
        v.p += (long long)(kb + v.cl) * v.ld;
        v.cs = INT_MAX;
        v.cl = 0;
    }
    return v;
}
__device__ __forceinline__ ZView view_from_row(ZView v, int kb) {
    if (v.rmap) {
        v.rmap += kb;
    } else if (v.rs >= kb) {
        v.p += kb;
        if (v.rs != INT_MAX) v.rs -= kb;
    } else {
        v.p += kb + v.rl;
        v.rs = INT_MAX;
        v.rl = 0;
    }
    return v;
}

// split-K pass on the tensor cores: blockIdx.z picks the k range [kb, kb + kchunk); the range's
// raw product (3M-combined, alpha = 1, no C) goes to the batch's workspace, laid out as the DFMA
// split pass writes it, for zgemm_reduce_kernel.  Every output element still sums its k range in
// MMA k-steps of 4 in order, so the result does not depend on n or on the tile shape.
template <int BM, int BN, int WM, int WN, int MINB>
__global__ void __launch_bounds__(32 * WM * WN, MINB)
zgemm_dmma_split_kernel(const GemmDesc* __restrict__ descs, int kchunk, z* work, long long pstride, int ldp, int ksplit) {
    extern __shared__ z dmma_smem[];
    __shared__ GemmDesc sd;
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(descs + blockIdx.y);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
        for (int w = threadIdx.x; w < (int)(sizeof(GemmDesc) / 8); w += 32 * WM * WN) dst[w] = src[w];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int kb = blockIdx.z * kchunk;
        sd.A = view_from_col(sd.A, kb);
        sd.B = view_from_row(sd.B, kb);
        sd.k = max(0, min(sd.k, kb + kchunk) - kb);
        sd.C = zview(nullptr, 1);
        sd.alpha = zmk(1.0, 0.0);
        sd.D = zout(work + ((long long)blockIdx.y * ksplit + blockIdx.z) * pstride, ldp);
    }
    __syncthreads();
    zgemm_tile_dmma<BM, BN, WM, WN>(sd, blockIdx.x, dmma_smem);
}

template <int BM, int BN, int WM, int WN, int MINB>
static cudaError_t launch_dmma_split(const GemmBatch& b, cudaStream_t s) {
    using Cfg = DmmaCfg<BM, BN, WM, WN>;
    auto kern = zgemm_dmma_split_kernel<BM, BN, WM, WN, MINB>;
    static DeviceAttrCache attr;
    {
        cudaError_t e = ensure_smem_attr(kern, Cfg::SMEM_BYTES, attr, true);
        if (e != cudaSuccess) return e;
    }
    if (b.count > 65535 || b.ksplit > 65535) return cudaErrorInvalidValue;
    const int tiles = ((b.max_m + BM - 1) / BM) * ((b.max_n + BN - 1) / BN);
    kern<<<dim3(tiles, b.count, b.ksplit), Cfg::NT, Cfg::SMEM_BYTES, s>>>(b.d_desc, b.kchunk, b.work, b.pstride,
                                                                        b.max_m, b.ksplit);
    note_launch();
    const long long elems = (long long)b.max_m * b.max_n;
    zgemm_reduce_kernel<<<dim3((unsigned)((elems + 255) / 256), b.count), 256, 0, s>>>(b.d_desc, b.work, b.pstride,
                                                                                     b.max_m, b.ksplit);
    note_launch();
    return cudaGetLastError();
}

template <int BM, int BN, int WM, int WN, int BK, int STAGES, int MINB>
__global__ void __launch_bounds__(32 * WM * WN, MINB) zgemm_dmma_kc_kernel(const GemmDesc* __restrict__ descs) {
    extern __shared__ z dmma_smem[];
    __shared__ GemmDesc sd;
    {
        const unsigned long long* src = reinterpret_cast<const unsigned long long*>(descs + blockIdx.y);
        unsigned long long* dst = reinterpret_cast<unsigned long long*>(&sd);
        for (int w = threadIdx.x; w < (int)(sizeof(GemmDesc) / 8); w += 32 * WM * WN) dst[w] = src[w];
    }
    __syncthreads();
    zgemm_tile_dmma_kc<BM, BN, WM, WN, BK, STAGES>(sd, blockIdx.x, dmma_smem);
}

template <int BM, int BN, int WM, int WN, int BK, int STAGES, int MINB>
static cudaError_t launch_dmma_kc(const GemmBatch& b, cudaStream_t s) {
    using Cfg = DmmaKcCfg<BM, BN, WM, WN, BK, STAGES>;
    auto kern = zgemm_dmma_kc_kernel<BM, BN, WM, WN, BK, STAGES, MINB>;
    static DeviceAttrCache attr;
    {
        cudaError_t e = ensure_smem_attr(kern, Cfg::SMEM_BYTES, attr, true);
        if (e != cudaSuccess) return e;
    }
    const int tiles = ((b.max_m + BM - 1) / BM) * ((b.max_n + BN - 1) / BN);
    for (int off = 0; off < b.count; off += 65535) {
        const int cnt = (b.count - off) < 65535 ? (b.count - off) : 65535;
        kern<<<dim3(tiles, cnt), Cfg::NT, Cfg::SMEM_BYTES, s>>>(b.d_desc + off);
        note_launch();
    }
    return cudaGetLastError();
}

// GEMM engine for the large problems: FP64 tensor-core MMA (default) or DFMA register tiles
// (RB_GEMM_ENGINE=dfma, read once; a tuning knob for comparisons)
static bool use_dmma() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("RB_GEMM_ENGINE");
        v = (e && std::strcmp(e, "dfma") == 0) ? 0 : 1;
    }
    return v == 1;
}

template <int BM, int BN, int TM, int TN, int BK, int STAGES, int MINB>
static cudaError_t launch_cfg(const GemmBatch& b, cudaStream_t s) {
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr size_t SMEM = DfmaCfg<BM, BN, BK, STAGES>::SMEM_BYTES;
    static DeviceAttrCache attr;
    if (SMEM > 48 * 1024) {
        cudaError_t e = ensure_smem_attr(zgemm_desc_kernel<BM, BN, TM, TN, BK, STAGES, MINB>, SMEM, attr);
        if (e != cudaSuccess) return e;
    }
    const int tiles = ((b.max_m + BM - 1) / BM) * ((b.max_n + BN - 1) / BN);
    for (int off = 0; off < b.count; off += 65535) {
        const int cnt = (b.count - off) < 65535 ? (b.count - off) : 65535;
        dim3 grid(tiles, cnt);
        zgemm_desc_kernel<BM, BN, TM, TN, BK, STAGES, MINB><<<grid, NT, SMEM, s>>>(b.d_desc + off);
        note_launch();
    }
    return cudaGetLastError();
}

template <int BM, int BN, int TM, int TN, int BK, int STAGES, int MINB>
static cudaError_t launch_split(const GemmBatch& b, cudaStream_t s) {
    constexpr int NT = (BM / TM) * (BN / TN);
    constexpr size_t SMEM = DfmaCfg<BM, BN, BK, STAGES>::SMEM_BYTES;
    static DeviceAttrCache attr;
    if (SMEM > 48 * 1024) {
        cudaError_t e = ensure_smem_attr(zgemm_split_kernel<BM, BN, TM, TN, BK, STAGES, MINB>, SMEM, attr);
        if (e != cudaSuccess) return e;
    }
    if (b.count > 65535 || b.ksplit > 65535) return cudaErrorInvalidValue;
    const int tiles = ((b.max_m + BM - 1) / BM) * ((b.max_n + BN - 1) / BN);
    zgemm_split_kernel<BM, BN, TM, TN, BK, STAGES, MINB><<<dim3(tiles, b.count, b.ksplit), NT, SMEM, s>>>(
        b.d_desc, b.kchunk, b.work, b.pstride, b.max_m, b.ksplit);
    note_launch();
    const long long elems = (long long)b.max_m * b.max_n;
    zgemm_reduce_kernel<<<dim3((unsigned)((elems + 255) / 256), b.count), 256, 0, s>>>(b.d_desc, b.work, b.pstride,
                                                                                     b.max_m, b.ksplit);
    note_launch();
    return cudaGetLastError();
}

// the kernel shape a batch runs on
enum class GemmShape { Dfma16, Dfma32, Dmma32, Dmma64, DmmaKc64, DmmaFixed, Dfma128x64, Dfma64 };
static GemmShape gemm_shape(const GemmBatch& b) {
    const int mm = b.max_m, nn = b.max_n;
    if (b.engine >= 0 && !b.fixed_order) return static_cast<GemmShape>(b.engine);
    // fixed-order batches (the solve) on the tensor cores: one tile shape, split-K planned from
    // count, m and k only; an element's sum runs over k in MMA steps of 4 in order whatever n is
    if (use_dmma() && b.fixed_order) return GemmShape::DmmaFixed;
    if (mm <= 16 && nn <= 16) return GemmShape::Dfma16;
    // FP64 tensor cores, small problems (both sides <= 192: the merges below 128x256 boxes):
    // 32x32 tiles of 4 warps, up to six CTAs per SM; measured 1.0-1.6x the 64x64 tile and
    // 1.3-1.4x the DFMA tiles on the merge shapes 16x48x16 .. 192x192x64
    if (use_dmma() && !b.fixed_order && mm <= 192 && nn <= 192) return GemmShape::Dmma32;
    // every DFMA shape sums an element's products in the same order, so the shape can follow the
    // available parallelism: small-n batches (the solve) that would leave SMs idle with 32x32
    // tiles take 16x16 tiles
    if (nn <= 32 && (long long)b.count * ((mm + 31) / 32) * ((nn + 31) / 32) < 2 * 148) return GemmShape::Dfma16;
    if (mm <= 32 || nn <= 32) return GemmShape::Dfma32;
    // FP64 tensor cores: 64x64 tiles of 8 warps, two CTAs per SM (16 warps to hide the MMA and
    // shared-memory latencies); measured faster than 128x64 tiles at one CTA per SM on every
    // merge shape from 64x256x64 x256 to 2048x4096x1024 x2
    if (use_dmma() && !b.fixed_order) {
        // contiguous-k batches with k >= 128: 32x32 warp tiles on stride-advanced copies,
        // measured 1.06-1.22x the tile above on the merge shapes 256x256x128 x256 ..
        // 2048x4096x1024 x2 (0.95x on 256x768x256 x8 and 128x512x128 x64, under two waves)
        if (b.kcontig && b.max_k >= 128) return GemmShape::DmmaKc64;
        return GemmShape::Dmma64;
    }
    // large problems: 8x4 complex register tile per thread (1.5 B of shared memory per DFMA)
    const bool big = mm >= 256 && nn >= 128 && (long long)b.count * ((mm + 127) / 128) * ((nn + 63) / 64) >= 148;
    return big ? GemmShape::Dfma128x64 : GemmShape::Dfma64;
}

long long gemm_plan_split(GemmBatch& b) {
    b.ksplit = 1;
    b.kchunk = 0;
    b.pstride = 0;
    // fixed-order batches run on tiles that share one summation order (the tensor-core tile, or
    // with RB_GEMM_ENGINE=dfma the DFMA tiles), so the split (and the rounding) depends on count,
    // m and k only
    if (!b.fixed_order || b.count == 0 || b.max_k < 128) return 0;
    // CTAs with one column tile (n-independent), against about four waves of two CTAs per SM
    const long long ctas = (long long)b.count * ((b.max_m + 15) / 16);
    long long sp = (4 * 148 + ctas - 1) / ctas;
    sp = std::min<long long>(sp, 16);
    sp = std::min<long long>(sp, b.max_k / 64);
    if (sp < 2) return 0;
    const int kc = (int)(((b.max_k + sp - 1) / sp + 7) / 8 * 8);
    b.kchunk = kc;
    b.ksplit = (b.max_k + kc - 1) / kc;
    if (b.ksplit < 2) {
        b.ksplit = 1;
        b.kchunk = 0;
        return 0;
    }
    b.pstride = (long long)b.max_m * b.max_n;
    return (long long)b.count * b.ksplit * b.pstride;
}

cudaError_t launch_gemm_reduce(const GemmBatch& b, int ksplit, long long pstride, cudaStream_t s) {
    const long long elems = (long long)b.max_m * b.max_n;
    if (b.count > 65535) return cudaErrorInvalidValue;
    zgemm_reduce_kernel<<<dim3((unsigned)((elems + 255) / 256), b.count), 256, 0, s>>>(b.d_desc, b.work, pstride,
                                                                                     b.max_m, ksplit);
    note_launch();
    return cudaGetLastError();
}

int gemm_engine_candidates(const GemmBatch& b, int* out) {
    int n = 0;
    if (b.fixed_order) return 0;
    out[n++] = (int)GemmShape::Dfma32;
    out[n++] = (int)GemmShape::Dfma64;
    if (use_dmma()) {
        out[n++] = (int)GemmShape::Dmma32;
        out[n++] = (int)GemmShape::Dmma64;
        if (b.kcontig) out[n++] = (int)GemmShape::DmmaKc64;
    }
    if (b.max_m >= 128) out[n++] = (int)GemmShape::Dfma128x64;
    return n;
}

const char* gemm_engine_name(int e) {
    switch (static_cast<GemmShape>(e)) {
        case GemmShape::Dfma16: return "dfma16";
        case GemmShape::Dfma32: return "dfma32";
        case GemmShape::Dmma32: return "dmma32";
        case GemmShape::Dmma64: return "dmma64";
        case GemmShape::DmmaKc64: return "dmma_kc64";
        case GemmShape::DmmaFixed: return "dmma_fixed";
        case GemmShape::Dfma128x64: return "dfma128x64";
        case GemmShape::Dfma64: return "dfma64";
    }
    return "?";
}

const char* gemm_stage_name(const GemmBatch& b) {
    const GemmShape sh = gemm_shape(b);
    // zgemm_tc: the contiguous-k tile (the large merge GEMMs); zgemm_tc_small: the other
    // tensor-core factor tiles; zgemm_tc_fixed: the solve's
    if (sh == GemmShape::DmmaFixed) return "zgemm_tc_fixed";
    if (sh == GemmShape::DmmaKc64) return "zgemm_tc";
    return (sh == GemmShape::Dmma64 || sh == GemmShape::Dmma32) ? "zgemm_tc_small" : "zgemm_dfma";
}

cudaError_t launch_gemm_batch(const GemmBatch& b, cudaStream_t s) {
    static_assert(sizeof(GemmDesc) % 8 == 0, "descriptor copy assumes 8-byte words");
    if (b.count == 0 || b.max_m == 0 || b.max_n == 0) return cudaSuccess;
    const GemmShape shape = gemm_shape(b);
    if (shape == GemmShape::DmmaFixed)
        return (b.ksplit > 1 && b.work) ? launch_dmma_split<32, 32, 2, 2, 6>(b, s) : launch_dmma<32, 32, 2, 2, 6>(b, s);
    if (b.ksplit > 1 && b.work) {
        if (shape == GemmShape::Dfma16) return launch_split<16, 16, 2, 2, 8, 6, 8>(b, s);
        if (shape == GemmShape::Dfma32) return launch_split<32, 32, 4, 2, 8, 4, 4>(b, s);
        if (shape == GemmShape::Dfma128x64) return launch_split<128, 64, 8, 4, 4, 4, 1>(b, s);
        if (shape == GemmShape::Dfma64) return launch_split<64, 64, 4, 4, 8, 4, 1>(b, s);
    }
    switch (shape) {
        case GemmShape::Dfma16: return launch_cfg<16, 16, 2, 2, 8, 6, 8>(b, s);
        case GemmShape::Dfma32: return launch_cfg<32, 32, 4, 2, 8, 4, 4>(b, s);
        case GemmShape::Dmma32:
        case GemmShape::DmmaFixed: return launch_dmma<32, 32, 2, 2, 6>(b, s);
        case GemmShape::Dmma64: return launch_dmma<64, 64, 2, 4, 2>(b, s);
        case GemmShape::DmmaKc64: return launch_dmma_kc<64, 64, 2, 2, 4, 8, 2>(b, s);
        case GemmShape::Dfma128x64: return launch_cfg<128, 64, 8, 4, 4, 4, 1>(b, s);
        case GemmShape::Dfma64: break;
    }
    return launch_cfg<64, 64, 4, 4, 8, 4, 1>(b, s);
}

}  // namespace rb
