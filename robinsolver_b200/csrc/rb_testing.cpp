// rb_testing.cpp -- test hooks of the GEMM and inversion engines, outside the drop-in C-ABI.
//
// rb_test_zgemm runs `count` complex GEMMs D_i = alpha A_i B_i + beta D_i (column-major, device
// pointers, plain strided views) on one engine, so that the tests can hold each engine against a
// host product directly:
//   engine 0: the FP64 launcher the FP64 path uses (tensor-core DMMA / DFMA tiles)
//   engine 1: the tcgen05 kernel of the mixed-precision levels in split TF32
//   engine 2: the tcgen05 kernel in int8 digit slices (the mixed-precision default)
// It allocates its descriptor array itself and synchronises; it returns 0, a negative RB_ERR_*
// code for bad arguments or CUDA failures, or the device status word's bits (> 0) when a kernel
// reported one.
#include <string>
#include <vector>

#include "robin_b200.h"
#include "rb_kernels.h"

using namespace rb;

// rb_test_zgemm_timed is the same call repeated `reps` times after one untimed run, and writes
// the mean device time of one batched launch in milliseconds to *ms (CUDA events; the engine's
// operand-split pass included).
static int test_zgemm(int engine, int m, int n, int k, const double* dA, long long lda, long long strideA,
                      const double* dB, long long ldb, long long strideB, double* dC, long long ldc,
                      long long strideC, double ar, double ai, double br, double bi, int count, int reps,
                      double* ms) {
    if (m <= 0 || n <= 0 || k <= 0 || count <= 0 || !dA || !dB || !dC || lda < m || ldb < k || ldc < m || reps < 0)
        return RB_ERR_INVALID;
    std::vector<GemmDesc> h(count);
    const z* A = reinterpret_cast<const z*>(dA);
    const z* B = reinterpret_cast<const z*>(dB);
    z* C = reinterpret_cast<z*>(dC);
    const bool use_beta = br != 0.0 || bi != 0.0;
    for (int i = 0; i < count; ++i) {
        GemmDesc& g = h[i];
        g = GemmDesc{};
        g.A = zview(A + i * strideA, lda);
        g.B = zview(B + i * strideB, ldb);
        g.C = use_beta ? zview(C + i * strideC, ldc) : zview(nullptr, 1);
        g.D = zout(C + i * strideC, ldc);
        g.alpha = zmk(ar, ai);
        g.beta = zmk(br, bi);
        g.m = m; g.n = n; g.k = k;
        g.nobeta_r0 = g.nobeta_r1 = 0;
    }
    GemmBatch b;
    b.count = count;
    b.max_m = m; b.max_n = n; b.max_k = k;
    b.kcontig = true;
    int* d_status = nullptr;
    if (cudaMalloc(&b.d_desc, sizeof(GemmDesc) * count) != cudaSuccess) return RB_ERR_CUDA;
    if (cudaMalloc(&d_status, sizeof(int)) != cudaSuccess) {
        cudaFree(b.d_desc);
        return RB_ERR_CUDA;
    }
    cudaError_t e = cudaSuccess;
    if (engine == 1 || engine == 2) {
        b.t5_engine = engine == 2 ? TC5_ENGINE_INT8 : TC5_ENGINE_TF32X3;
        const size_t pb = tc5_plane_bytes(b);
        if (pb) e = cudaMalloc(&b.t5_planes, pb);
        b.t5_plane_cap = pb;
    }
    auto run = [&]() { return engine != 0 ? launch_gemm_tc5(b, d_status, 0) : launch_gemm_batch(b, 0); };
    int rc = RB_OK;
    if (e == cudaSuccess) e = cudaMemcpy(b.d_desc, h.data(), sizeof(GemmDesc) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_status, 0, sizeof(int));
    if (e == cudaSuccess) e = run();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess && reps > 0) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        if (e == cudaSuccess) e = cudaEventRecord(e0, 0);
        for (int r = 0; r < reps && e == cudaSuccess; ++r) e = run();
        if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        float t = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
        if (e == cudaSuccess && ms) *ms = (double)t / reps;
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
    int st = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        set_thread_error((std::string("rb_test_zgemm: ") + cudaGetErrorString(e)).c_str());
        rc = RB_ERR_CUDA;
    } else {
        rc = st;
    }
    cudaFree(b.d_desc);
    cudaFree(d_status);
    if (b.t5_planes) cudaFree(b.t5_planes);
    return rc;
}

extern "C" int rb_test_zgemm(int engine, int m, int n, int k, const double* dA, long long lda, long long strideA,
                             const double* dB, long long ldb, long long strideB, double* dC, long long ldc,
                             long long strideC, double ar, double ai, double br, double bi, int count) {
    return test_zgemm(engine, m, n, k, dA, lda, strideA, dB, ldb, strideB, dC, ldc, strideC, ar, ai, br, bi, count,
                      0, nullptr);
}

extern "C" int rb_test_zgemm_timed(int engine, int m, int n, int k, const double* dA, long long lda,
                                   long long strideA, const double* dB, long long ldb, long long strideB, double* dC,
                                   long long ldc, long long strideC, double ar, double ai, double br, double bi,
                                   int count, int reps, double* ms) {
    return test_zgemm(engine, m, n, k, dA, lda, strideA, dB, ldb, strideB, dC, ldc, strideC, ar, ai, br, bi, count,
                      reps, ms);
}

// rb_test_zinvert inverts `count` complex m x m matrices in place (column-major, device pointers,
// A_i = dA + i * stride, leading dimension ld) with the batched Gauss-Jordan kernels of the
// factorization, `reps` times in a row (each call inverts the previous result), and writes the
// mean device time of one batched inversion in milliseconds to *ms (may be null).  It returns 0,
// a negative RB_ERR_* code, or the device status word's bits (> 0) when a kernel reported one
// (1: a zero pivot; 2: a resident CTA gave up waiting).
extern "C" int rb_test_zinvert(int m, int count, double* dA, long long ld, long long stride, int reps, double* ms) {
    if (m <= 0 || count <= 0 || reps <= 0 || !dA || ld < m || (count > 1 && stride < ld * m)) return RB_ERR_INVALID;
    z* A = reinterpret_cast<z*>(dA);
    const long long ws = gj_workspace_elems(m);
    std::vector<GJDesc> h(count);
    GJDesc* d_desc = nullptr;
    int* d_ipiv = nullptr;
    int* d_status = nullptr;
    z* d_work = nullptr;
    auto release = [&]() {
        cudaFree(d_desc);
        cudaFree(d_ipiv);
        cudaFree(d_status);
        cudaFree(d_work);
    };
    cudaError_t e = cudaMalloc(&d_desc, sizeof(GJDesc) * count);
    if (e == cudaSuccess) e = cudaMalloc(&d_ipiv, sizeof(int) * (size_t)m * count);
    if (e == cudaSuccess) e = cudaMalloc(&d_status, sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&d_work, sizeof(z) * (size_t)std::max<long long>(1, ws * count));
    if (e != cudaSuccess) {
        release();
        set_thread_error((std::string("rb_test_zinvert: ") + cudaGetErrorString(e)).c_str());
        return RB_ERR_CUDA;
    }
    for (int i = 0; i < count; ++i) {
        h[i].A = A + (long long)i * stride;
        h[i].ld = ld;
        h[i].ipiv = d_ipiv + (long long)i * m;
        h[i].Zb = d_work + (long long)i * ws;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    e = cudaMemcpy(d_desc, h.data(), sizeof(GJDesc) * count, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_status, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaEventRecord(e0, 0);
    for (int r = 0; r < reps && e == cudaSuccess; ++r) e = gj_invert_batch(d_desc, count, m, d_work, d_status, 0);
    if (e == cudaSuccess) e = cudaEventRecord(e1, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    float t = 0.0f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
    int st = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    release();
    if (e != cudaSuccess) {
        set_thread_error((std::string("rb_test_zinvert: ") + cudaGetErrorString(e)).c_str());
        return RB_ERR_CUDA;
    }
    if (ms) *ms = t / reps;
    return st;
}
