// C ABI of the B200 propagator library (see include/crysscft_b200.h).
//
// Host side: solver objects holding the per-axis operators (built once per
// (cell, ds) in long double, stored FP64 and FP32 on the device), the
// triplet/contour launchers, and the AB-diblock iteration context whose whole
// iteration is captured once into a CUDA graph and replayed.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/crysscft_b200.h"
#include "axis_dmma.cuh"
#include "axis_fft.cuh"
#include "axis_kernels.cuh"
#include "contour_kernel.cuh"
#include "contour_batch.cuh"
#include "contour_cluster_f32.cuh"
#include "contour_kernel_f32.cuh"
#include "field_kernels.cuh"
#include "operators.h"
#include "stress_kernels.cuh"

using namespace crysscft;

namespace {

thread_local std::string g_last_error = "";

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? SCFT_ERR_ALLOC : SCFT_ERR_CUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

#define CKR(call)                          \
    do {                                   \
        int r_ = (call);                   \
        if (r_ != SCFT_OK) return r_;      \
    } while (0)

// L2 eviction priorities on the tensor-core axis passes (axis_dmma.cuh); off with
// CRYSSCFT_L2_HINTS=0 (read once).
int l2_hints_enabled() {
    static const int on = [] {
        const char* e = getenv("CRYSSCFT_L2_HINTS");
        return (e && e[0] == '0') ? 0 : 1;
    }();
    return on;
}

// TMA descriptor encoder of the driver (cuTensorMapEncodeTiled), resolved once.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor map of an n^3 FP64 field (slots > 0: a contour store of `slots` fields) as n x n
// tiles in 8-column panels: dims (z % 8, row, z / 8, tile[, slot]), box (8, n, n / 8, 1[, 1]),
// so a box lands in shared memory as [z / 8][row][z % 8].  plane: row = y, tile = x;
// else (slab): row = x, tile = y.
int encode_panel_map(CUtensorMap* m, const void* base, int n, long long slots, bool plane, bool fp64 = true) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc) return fail(SCFT_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    if (reinterpret_cast<uintptr_t>(base) % 16) return fail(SCFT_ERR_INVALID_ARG, "TMA base not 16-byte aligned");
    if (n % 8 || n > 256) return fail(SCFT_ERR_INVALID_ARG, "panel tiles need n a multiple of 8, at most 256");
    const cuuint64_t es = fp64 ? 8 : 4, N = (cuuint64_t)n;
    cuuint64_t dims[5] = {8, N, N / 8, N, (cuuint64_t)(slots > 0 ? slots : 1)};
    cuuint64_t strides[4] = {plane ? N * es : N * N * es, 8 * es, plane ? N * N * es : N * es, N * N * N * es};
    cuuint32_t box[5] = {8u, (cuuint32_t)n, (cuuint32_t)(n / 8), 1u, 1u};
    cuuint32_t estr[5] = {1u, 1u, 1u, 1u, 1u};
    const CUresult r = enc(m, fp64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                           slots > 0 ? 5u : 4u, const_cast<void*>(base), dims,
                           strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(SCFT_ERR_CUDA, "cuTensorMapEncodeTiled (panel tiles) failed (" + std::to_string((int)r) + ")");
    return SCFT_OK;
}

// Flags of the alternating kernels at n^3: [chain][plane|slab][consumer][producer] exchange
// flags, then [chain][unit] landed-store counts of the fused phi sums.
static size_t alt_flag_count(int nx) { return (size_t)4 * nx * nx + (size_t)2 * nx; }

// Zero device memory before any of the library's streams uses it.  cudaMemset runs on the
// legacy default stream and may return before it has run, and the library's streams are
// non-blocking (they do not wait for the legacy stream), so wait for it here.
static int zero_device(void* p, size_t bytes) {
    CK(cudaMemset(p, 0, bytes));
    CK(cudaStreamSynchronize(0));
    return SCFT_OK;
}

// Host-to-device upload for set-up data (operators, tables, task lists).  A cudaMemcpy from
// pageable host memory may return once the data is staged, before it has reached the
// device, and the kernels that read it run on non-blocking streams: wait for the copy.
static int upload(void* dst, const void* src, size_t bytes) {
    CK(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(0));
    return SCFT_OK;
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    int alloc(size_t count) {
        release();
        if (count == 0) return SCFT_OK;
        cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            return fail(SCFT_ERR_ALLOC, std::string("cudaMalloc(") + std::to_string(count * sizeof(T)) +
                                            " bytes): " + cudaGetErrorString(e));
        }
        n = count;
        return SCFT_OK;
    }
};

struct OpsSet {
    DevBuf<double> d_op[3], d_opT[3];
    DevBuf<float> f_op[3], f_opT[3];
    // packed per-axis operators for the persistent contour kernel (FP64): for an
    // even/odd axis E then O (h x h, leading dimension h+4), else A (n x n, n+4)
    std::vector<double> h_packed;
    DevBuf<double> d_packed;
    // two even/odd levels (PMMM, n = 64 or 128 on every axis): per axis [EE | EO | O]
    // (AxisShapeEO2), x then y then z
    std::vector<double> h_packed2;
    DevBuf<double> d_packed2;
    bool eo2 = false;
    int eo[3] = {0, 0, 0}, off[3] = {0, 0, 0}, ld[3] = {0, 0, 0}, half[3] = {0, 0, 0};
    int total = 0;
    // FP32 precision form: per axis [hi][lo] TF32 split parts, each E,O (even/odd) or A
    std::vector<float> h_packed_f32;
    DevBuf<float> f_packed;
    int eo_f32[3] = {0, 0, 0};
    // FP32 precision form on clusters (64-point even/odd axes): per axis the fp16 parts
    // [E_hi | E_lo | O_hi | O_lo] in the tensor cores' K-major operand layout
    std::vector<uint16_t> h_packed_h16;
    DevBuf<__half> h16_packed;
    int h16_axes = 0;  // axes packed (3: the cluster kernel can run)
    // FFT form of the FP64 axis passes (axis_fft.cuh): per axis the transform length (0: the
    // axis has none), the extension (0 P1, 1 PMMM mirror, 2 3m interleave), the spectrum g
    // (1/NF included) and the NF twiddles
    int fft_nf[3] = {0, 0, 0}, fft_ext[3] = {0, 0, 0};
    DevBuf<double> d_fft_g[3];
    DevBuf<double2> d_fft_tw[3];
    DevBuf<float> f_fft_g[3];   // the same tables rounded to FP32 (precision form)
    DevBuf<float2> f_fft_tw[3];
    // cell-length derivatives dA/dL of the three axis operators (built on first use)
    DevBuf<double> d_dop[3], d_dopT[3];
    bool have_dop = false;
    // an operator that is a sum of Kronecker products (3m with mirror translations):
    // this set holds term 0, `more` the others (their d_op/f_op/d_dop only); the packed
    // operators and the persistent contour kernels serve single-term operators only
    int nterms = 1;
    std::vector<std::unique_ptr<OpsSet>> more;
    OpsSet* term(int t) { return t == 0 ? this : more[(size_t)t - 1].get(); }
};

// Round an FP32 value to the TF32 format (10 explicit mantissa bits), to nearest with
// ties away from zero; the result is an FP32 value whose low 13 mantissa bits are 0.
float round_to_tf32(float x) {
    uint32_t u;
    std::memcpy(&u, &x, sizeof(u));
    if ((u & 0x7f800000u) != 0x7f800000u) {
        u += 0x1000u;
        u &= 0xffffe000u;
    }
    float r;
    std::memcpy(&r, &u, sizeof(r));
    return r;
}

// Append one axis operator to the FP32 packed buffer as TF32 hi/lo parts:
// hi = tf32(a), lo = tf32(a - hi) evaluated from the long double value.
void pack_operator_f32(const std::vector<long double>& A, int n, OpsSet& s, int axis) {
    bool centro = (n % 32 == 0);
    for (int i = 0; centro && i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const long double a = A[(size_t)i * n + j], b = A[(size_t)(n - 1 - i) * n + (n - 1 - j)];
            if (fabsl(a - b) > 1e-17L * (1.0L + fabsl(a))) { centro = false; break; }
        }
    s.eo_f32[axis] = centro ? 1 : 0;
    const int K = centro ? n / 2 : n, ld = K + 4;
    const size_t part = centro ? 2 * (size_t)K * ld : (size_t)n * ld;
    const size_t base = s.h_packed_f32.size();
    s.h_packed_f32.resize(base + 2 * part, 0.0f);
    float* hi = s.h_packed_f32.data() + base;
    float* lo = hi + part;
    auto put = [&](size_t idx, long double v) {
        const float h = round_to_tf32((float)v);
        hi[idx] = h;
        lo[idx] = round_to_tf32((float)(v - (long double)h));
    };
    for (int i = 0; i < (centro ? K : n); ++i)
        for (int j = 0; j < K; ++j) {
            if (centro) {
                const long double a = A[(size_t)i * n + j], b = A[(size_t)i * n + (n - 1 - j)];
                put((size_t)i * ld + j, (a + b) / 2);
                put((size_t)K * ld + (size_t)i * ld + j, (a - b) / 2);
            } else {
                put((size_t)i * ld + j, A[(size_t)i * n + j]);
            }
        }
}

// fp16 value of v rounded to nearest (ties to even), as its 16-bit pattern; v is finite
// and below 65504 in magnitude (operator entries and their 2^12-scaled residuals)
uint16_t half_bits_rn(long double v) {
    // quantum of the fp16 grid at |v|: 2^(e - 10) for normal values, 2^-24 below 2^-14
    const long double a = fabsl(v);
    int e = 0;
    if (a > 0) frexpl(a, &e);  // a = m 2^e, m in [0.5, 1): the leading bit is 2^(e - 1)
    const int lead = a > 0 ? e - 1 : -14;
    const long double quantum = ldexpl(1.0L, (lead < -14 ? -14 : lead) - 10);
    const long double qv = nearbyintl(v / quantum) * quantum;  // round half to even (default mode)
    return __half_as_ushort(__float2half_rn((float)qv));          // exact: qv lies on the fp16 grid
}

// Append one axis operator (64 x 64, centrosymmetric) as the fp16 operator parts of the
// cluster kernel: E = (A[i][j] + A[i][63-j]) / 2, O = (A[i][j] - A[i][63-j]) / 2 (32 x 32),
// each split into hi = fp16(x) and lo = fp16((x - hi) 2^12), stored in the canonical K-major
// layout of a tcgen05 operand (row i = output, k = j: element (i, j) at byte
// (i / 8) 512 + (j / 8) 128 + (i % 8) 16 + (j % 8) 2).  Returns false (nothing appended)
// for other operators.
bool pack_operator_h16(const std::vector<long double>& A, int n, OpsSet& s) {
    if (n != kClN) return false;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const long double a = A[(size_t)i * n + j], b = A[(size_t)(n - 1 - i) * n + (n - 1 - j)];
            if (fabsl(a - b) > 1e-17L * (1.0L + fabsl(a))) return false;
            if (!(fabsl(a) < 8.0L)) return false;  // fp16 range with room for the even/odd sums
        }
    const int h = n / 2;
    const size_t base = s.h_packed_h16.size();
    s.h_packed_h16.resize(base + (size_t)kClOpAxis, 0);
    uint16_t* out = s.h_packed_h16.data() + base;
    auto at = [](int i, int j) { return (size_t)((i / 8) * 256 + (j / 8) * 64 + (i % 8) * 8 + (j % 8)); };
    for (int i = 0; i < h; ++i)
        for (int j = 0; j < h; ++j) {
            const long double a = A[(size_t)i * n + j], b = A[(size_t)i * n + (n - 1 - j)];
            const long double parts[2] = {(a + b) / 2, (a - b) / 2};
            for (int m = 0; m < 2; ++m) {
                const uint16_t hi = half_bits_rn(parts[m]);
                const long double hv = (long double)__half2float(__ushort_as_half(hi));
                out[(size_t)(2 * m) * kClOpMat + at(i, j)] = hi;
                out[(size_t)(2 * m + 1) * kClOpMat + at(i, j)] = half_bits_rn((parts[m] - hv) * 4096.0L);
            }
        }
    ++s.h16_axes;
    return true;
}

// Tables of the FFT axis pass of one axis: the spectrum of the circulant,
// g_k = exp(-ds (2 pi min(k, NF - k) / L)^2) / NF (the factor of K in src/solver_p1.h:149-165,
// src/solver_Pmmm.h:166-179, src/solver_3m.h:197-231, with the transforms' normalisation),
// and the twiddles exp(-2 pi i m / NF), both in long double rounded once.
int upload_fft_tables(OpsSet& s, int axis, int nf, int ext, long double L, long double ds) {
    static const long double kPiL = 3.141592653589793238462643383279502884L;
    std::vector<double> g((size_t)nf);
    std::vector<double2> tw((size_t)nf);
    for (int k = 0; k < nf; ++k) {
        const long double kk = 2.0L * kPiL * (long double)(k < nf - k ? k : nf - k) / L;
        g[(size_t)k] = (double)(expl(-ds * kk * kk) / (long double)nf);
        const long double a = -2.0L * kPiL * (long double)k / (long double)nf;
        tw[(size_t)k] = make_double2((double)cosl(a), (double)sinl(a));
    }
    CKR(s.d_fft_g[axis].alloc((size_t)nf));
    CKR(s.d_fft_tw[axis].alloc((size_t)nf));
    CKR(upload(s.d_fft_g[axis].p, g.data(), g.size() * sizeof(double)));
    CKR(upload(s.d_fft_tw[axis].p, tw.data(), tw.size() * sizeof(double2)));
    std::vector<float> gf((size_t)nf);
    std::vector<float2> twf((size_t)nf);
    for (int k = 0; k < nf; ++k) {
        gf[(size_t)k] = (float)g[(size_t)k];
        twf[(size_t)k] = make_float2((float)tw[(size_t)k].x, (float)tw[(size_t)k].y);
    }
    CKR(s.f_fft_g[axis].alloc((size_t)nf));
    CKR(s.f_fft_tw[axis].alloc((size_t)nf));
    CKR(upload(s.f_fft_g[axis].p, gf.data(), gf.size() * sizeof(float)));
    CKR(upload(s.f_fft_tw[axis].p, twf.data(), twf.size() * sizeof(float2)));
    s.fft_nf[axis] = nf;
    s.fft_ext[axis] = ext;
    return SCFT_OK;
}

template <typename R>
using AxisFftFn = void (*)(const AxisFftPass<R>);

// The FFT pass kernel of an axis of length n with transform length nf and extension ext.
template <typename R>
AxisFftFn<R> axis_fft_kernel_for(int n, int nf, int ext, size_t* smem) {
#define CRYSSCFT_FFT_CASE(N_, NF_, EXT_)                         \
    if (n == N_ && nf == NF_ && ext == EXT_) {                   \
        *smem = FftShape<N_, NF_, EXT_, R>::SMEM;                \
        return axis_fft_kernel<N_, NF_, EXT_, R>;                \
    }
    CRYSSCFT_FFT_CASE(64, 64, 0)
    CRYSSCFT_FFT_CASE(128, 128, 0)
    CRYSSCFT_FFT_CASE(256, 256, 0)
    CRYSSCFT_FFT_CASE(32, 64, 1)
    CRYSSCFT_FFT_CASE(64, 128, 1)
    CRYSSCFT_FFT_CASE(128, 256, 1)
    CRYSSCFT_FFT_CASE(32, 64, 2)
    CRYSSCFT_FFT_CASE(64, 128, 2)
    CRYSSCFT_FFT_CASE(128, 256, 2)
#undef CRYSSCFT_FFT_CASE
    return nullptr;
}

// Which form runs the per-axis passes: CRYSSCFT_AXIS_FORM=fft or =dense forces one (for
// measurements and tests); by default the FFT passes run wherever they exist except where
// the tensor-core passes were measured faster (scft_solver_s::tensor_axis_passes: PMMM
// grids they cover, and P1 iterations).  Per triplet on one B200: 256-point P1 axes 0.28 ms
// by FFT against 2.99 ms by the SIMT GEMMs; 128-point PMMM axes 65 us by FFT against 56 us
// by DMMA.
int axis_form_override() {
    const char* e = getenv("CRYSSCFT_AXIS_FORM");
    return !e ? 0 : (e[0] == 'f' ? 1 : (e[0] == 'd' ? 2 : 0));
}

// Append one axis operator to the packed buffer, in even/odd form when A is
// centrosymmetric (A[n-1-i][n-1-j] == A[i][j]) and n is a multiple of 16.
void pack_operator(const std::vector<long double>& A, int n, OpsSet& s, int axis) {
    bool centro = (n % 16 == 0);
    for (int i = 0; centro && i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const long double a = A[(size_t)i * n + j], b = A[(size_t)(n - 1 - i) * n + (n - 1 - j)];
            if (fabsl(a - b) > 1e-17L * (1.0L + fabsl(a))) { centro = false; break; }
        }
    s.off[axis] = (int)s.h_packed.size();
    if (centro) {
        const int h = n / 2, ld = h + 4;
        s.eo[axis] = 1;
        s.ld[axis] = ld;
        s.half[axis] = h * ld;
        s.h_packed.resize(s.h_packed.size() + 2 * (size_t)h * ld, 0.0);
        double* E = s.h_packed.data() + s.off[axis];
        double* O = E + (size_t)h * ld;
        for (int i = 0; i < h; ++i)
            for (int j = 0; j < h; ++j) {
                const long double a = A[(size_t)i * n + j], b = A[(size_t)i * n + (n - 1 - j)];
                E[(size_t)i * ld + j] = (double)((a + b) / 2);
                O[(size_t)i * ld + j] = (double)((a - b) / 2);
            }
    } else {
        const int ld = n + 4;
        s.eo[axis] = 0;
        s.ld[axis] = ld;
        s.half[axis] = 0;
        s.h_packed.resize(s.h_packed.size() + (size_t)n * ld, 0.0);
        double* D = s.h_packed.data() + s.off[axis];
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) D[(size_t)i * ld + j] = (double)A[(size_t)i * n + j];
    }
    s.total = (int)s.h_packed.size();
}

// Append one axis operator in the two-level even/odd form when its even half is itself
// centrosymmetric (PMMM) and n is 64 (whole-contour kernel) or 128 (axis passes); returns
// false (and appends nothing) otherwise.
bool pack_operator_eo2(const std::vector<long double>& A, int n, OpsSet& s) {
    if (n != 64 && n != 128) return false;
    const int h = n / 2, h2 = n / 4;
    std::vector<long double> E((size_t)h * h), O((size_t)h * h);
    for (int i = 0; i < h; ++i)
        for (int j = 0; j < h; ++j) {
            const long double a = A[(size_t)i * n + j], b = A[(size_t)i * n + (n - 1 - j)];
            E[(size_t)i * h + j] = (a + b) / 2;
            O[(size_t)i * h + j] = (a - b) / 2;
            if (fabsl(a - A[(size_t)(n - 1 - i) * n + (n - 1 - j)]) > 1e-17L * (1.0L + fabsl(a))) return false;
        }
    for (int i = 0; i < h; ++i)
        for (int j = 0; j < h; ++j) {
            const long double a = E[(size_t)i * h + j], b = E[(size_t)(h - 1 - i) * h + (h - 1 - j)];
            if (fabsl(a - b) > 1e-17L * (1.0L + fabsl(a))) return false;
        }
    const int ld2 = h2 + 4, ld = h + 4;
    const size_t base = s.h_packed2.size();
    s.h_packed2.resize(base + 2 * (size_t)h2 * ld2 + (size_t)h * ld, 0.0);
    double* EE = s.h_packed2.data() + base;
    double* EO = EE + (size_t)h2 * ld2;
    double* OO = EO + (size_t)h2 * ld2;
    for (int i = 0; i < h2; ++i)
        for (int j = 0; j < h2; ++j) {
            const long double a = E[(size_t)i * h + j], b = E[(size_t)i * h + (h - 1 - j)];
            EE[(size_t)i * ld2 + j] = (double)((a + b) / 2);
            EO[(size_t)i * ld2 + j] = (double)((a - b) / 2);
        }
    for (int i = 0; i < h; ++i)
        for (int j = 0; j < h; ++j) OO[(size_t)i * ld + j] = (double)O[(size_t)i * h + j];
    return true;
}

int upload_operator(const std::vector<long double>& A, int n, OpsSet& s, int axis) {
    std::vector<double> d((size_t)n * n), dt((size_t)n * n);
    std::vector<float> f((size_t)n * n), ft((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const long double v = A[(size_t)i * n + j];
            d[(size_t)i * n + j] = (double)v;
            dt[(size_t)j * n + i] = (double)v;
            f[(size_t)i * n + j] = (float)v;
            ft[(size_t)j * n + i] = (float)v;
        }
    const size_t nn = (size_t)n * n;
    CKR(s.d_op[axis].alloc(nn));
    CKR(s.d_opT[axis].alloc(nn));
    CKR(s.f_op[axis].alloc(nn));
    CKR(s.f_opT[axis].alloc(nn));
    CKR(upload(s.d_op[axis].p, d.data(), nn * sizeof(double)));
    CKR(upload(s.d_opT[axis].p, dt.data(), nn * sizeof(double)));
    CKR(upload(s.f_op[axis].p, f.data(), nn * sizeof(float)));
    CKR(upload(s.f_opT[axis].p, ft.data(), nn * sizeof(float)));
    return SCFT_OK;
}

int grid_blocks(long long M, int threads) {
    long long b = (M + threads - 1) / threads;
    if (b > 148LL * 8) b = 148LL * 8;
    if (b < 1) b = 1;
    return (int)b;
}

// ---------------------------------------------------------------------------
// axis-pass launchers
// ---------------------------------------------------------------------------
template <typename T, int BM>
cudaError_t launch_strided_bm(const AxisPass<T>& p, int nchain, cudaStream_t st) {
    constexpr int BN = 64, BK = 16, TM = 4, TN = 4;
    dim3 grid((unsigned)((p.inner + BN - 1) / BN), (unsigned)((p.n + BM - 1) / BM),
              (unsigned)(p.outer * nchain));
    axis_strided_kernel<T, BM, BN, BK, TM, TN><<<grid, (BM / TM) * (BN / TN), 0, st>>>(p);
    return cudaGetLastError();
}
template <typename T, int BN>
cudaError_t launch_contig_bn(const AxisPass<T>& p, int nchain, cudaStream_t st) {
    constexpr int BM = 64, BK = 16, TM = 4, TN = 4;
    dim3 grid((unsigned)((p.n + BN - 1) / BN), (unsigned)((p.outer + BM - 1) / BM), (unsigned)nchain);
    axis_contig_kernel<T, BM, BN, BK, TM, TN><<<grid, (BM / TM) * (BN / TN), 0, st>>>(p);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_axis(const AxisPass<T>& p, int nchain, bool contiguous, cudaStream_t st) {
    if (contiguous) {
        if (p.n <= 16) return launch_contig_bn<T, 16>(p, nchain, st);
        if (p.n <= 32) return launch_contig_bn<T, 32>(p, nchain, st);
        return launch_contig_bn<T, 64>(p, nchain, st);
    }
    if (p.n <= 16) return launch_strided_bm<T, 16>(p, nchain, st);
    if (p.n <= 32) return launch_strided_bm<T, 32>(p, nchain, st);
    return launch_strided_bm<T, 64>(p, nchain, st);
}

using AxisDmmaFn = void (*)(const AxisPassD);

// The FP64 tensor-core axis pass for a cubic grid of side n (96 or 128); nullptr if none.
// eo2: the operators are in the two-level even/odd form (AxisShapeEO2, n = 128).
AxisDmmaFn axis_dmma_kernel_for(int n, int eo, int ax, size_t* smem, bool eo2 = false) {
    if (eo2 && eo && n == 128) {
        *smem = AxisDmmaShape<128, true, true>::SMEM;
        return ax == 0 ? axis_dmma_kernel<128, true, 0, true>
                       : (ax == 1 ? axis_dmma_kernel<128, true, 1, true> : axis_dmma_kernel<128, true, 2, true>);
    }
#define CRYSSCFT_AXD(N, E)                                            \
    {                                                                 \
        *smem = AxisDmmaShape<N, E>::SMEM;                            \
        return ax == 0 ? axis_dmma_kernel<N, E, 0>                    \
                       : (ax == 1 ? axis_dmma_kernel<N, E, 1> : axis_dmma_kernel<N, E, 2>); \
    }
    if (n == 128) {
        if (eo) CRYSSCFT_AXD(128, true) else CRYSSCFT_AXD(128, false)
    }
    if (n == 96) {
        if (eo) CRYSSCFT_AXD(96, true) else CRYSSCFT_AXD(96, false)
    }
#undef CRYSSCFT_AXD
    return nullptr;
}

using AxisTf32Fn = void (*)(const AxisPassF);

// The FP32 (3xTF32) axis pass for a cubic grid of side n (96 or 128); nullptr if none.
// *op_stride: floats between consecutive axes' operators in the packed FP32 buffer.
AxisTf32Fn axis_tf32_kernel_for(int n, int eo, int ax, size_t* smem, size_t* op_stride) {
#define CRYSSCFT_AXF(N, E)                                                                    \
    {                                                                                         \
        *smem = AxisTf32Shape<N, E>::SMEM;                                                    \
        *op_stride = AxisShapeF<N, E>::SIZE;                                                  \
        return ax == 0 ? axis_tf32_kernel<N, E, 0>                                            \
                       : (ax == 1 ? axis_tf32_kernel<N, E, 1> : axis_tf32_kernel<N, E, 2>);   \
    }
    if (n == 128) {
        if (eo) CRYSSCFT_AXF(128, true) else CRYSSCFT_AXF(128, false)
    }
    if (n == 96) {
        if (eo) CRYSSCFT_AXF(96, true) else CRYSSCFT_AXF(96, false)
    }
#undef CRYSSCFT_AXF
    return nullptr;
}

using ContourFn = void (*)(const ContourArgs);

// The alternating-layout contour kernel for cubic grids whose four tiles and operators
// fit in shared memory; nullptr when there is none.
using ContourFnF = void (*)(const ContourArgsF);

// The FP32 (3xTF32) alternating-layout kernel for a cubic grid; nullptr when there is none.
ContourFnF contour_alt_kernel_f32_for(int n, int eo, size_t* smem) {
#define CRYSSCFT_ALTF(N, E)                    \
    {                                          \
        *smem = AltShapeF<N, E>::SMEM;         \
        return contour_alt_kernel_f32<N, E>;   \
    }
    if (eo) {
        switch (n) {
            case 32: CRYSSCFT_ALTF(32, true)
            case 64: CRYSSCFT_ALTF(64, true)
            default: break;
        }
    } else {
        switch (n) {
            case 16: CRYSSCFT_ALTF(16, false)
            case 32: CRYSSCFT_ALTF(32, false)
            case 48: CRYSSCFT_ALTF(48, false)
            case 64: CRYSSCFT_ALTF(64, false)
            default: break;
        }
    }
#undef CRYSSCFT_ALTF
    return nullptr;
}

ContourFn contour_alt_kernel_for(int n, int eo, size_t* smem, bool eo2 = false) {
    if (eo2 && eo && n == 64) {
        *smem = AltShape<64, true, true>::SMEM;
        return contour_alt_kernel<64, true, true>;
    }
#define CRYSSCFT_ALT(N, E)                     \
    {                                          \
        *smem = AltShape<N, E>::SMEM;          \
        return contour_alt_kernel<N, E>;       \
    }
    if (eo) {
        switch (n) {
            case 16: CRYSSCFT_ALT(16, true)
            case 32: CRYSSCFT_ALT(32, true)
            case 48: CRYSSCFT_ALT(48, true)
            case 64: CRYSSCFT_ALT(64, true)
            default: break;
        }
    } else {
        switch (n) {
            case 8: CRYSSCFT_ALT(8, false)
            case 16: CRYSSCFT_ALT(16, false)
            case 24: CRYSSCFT_ALT(24, false)
            case 32: CRYSSCFT_ALT(32, false)
            case 40: CRYSSCFT_ALT(40, false)
            case 48: CRYSSCFT_ALT(48, false)
            case 56: CRYSSCFT_ALT(56, false)
            default: break;
        }
    }
#undef CRYSSCFT_ALT
    return nullptr;
}

// The compile-time specialised contour kernel for cubic grids (all axes even/odd, or
// all full), else the runtime-generic one.
ContourFn contour_kernel_for(int nx, int ny, int nz, const int eo[3]) {
    if (nx == ny && ny == nz && eo[0] == eo[1] && eo[1] == eo[2]) {
        if (eo[0]) {
            switch (nx) {
                case 16: return contour_kernel_ct<16, 16, 16, true, true, true>;
                case 32: return contour_kernel_ct<32, 32, 32, true, true, true>;
                case 48: return contour_kernel_ct<48, 48, 48, true, true, true>;
                case 64: return contour_kernel_ct<64, 64, 64, true, true, true>;
                default: break;
            }
        } else {
            switch (nx) {
                case 8: return contour_kernel_ct<8, 8, 8, false, false, false>;
                case 16: return contour_kernel_ct<16, 16, 16, false, false, false>;
                case 24: return contour_kernel_ct<24, 24, 24, false, false, false>;
                case 32: return contour_kernel_ct<32, 32, 32, false, false, false>;
                case 40: return contour_kernel_ct<40, 40, 40, false, false, false>;
                case 48: return contour_kernel_ct<48, 48, 48, false, false, false>;
                case 56: return contour_kernel_ct<56, 56, 56, false, false, false>;
                case 64: return contour_kernel_ct<64, 64, 64, false, false, false>;
                default: break;
            }
        }
    }
    return contour_kernel_f64;
}

}  // namespace

// ---------------------------------------------------------------------------
// solver
// ---------------------------------------------------------------------------
struct scft_solver_s {
    int kind = 0;
    int precision = SCFT_FP64;
    int device = 0;
    int users = 0;                 // iteration contexts (scft_diblock_t) built on this solver
    bool destroy_pending = false;  // scft_solver_destroy was called while users > 0
    int sms = 0;                   // multiprocessors of `device` (queried on first use)
    size_t axis_dmma_smem_set = 0; // dynamic shared memory granted to the tensor-core axis passes
    const void* axis_dmma_fn_set = nullptr;  // ... and to which kernel family (z pass)
    size_t axis_tf32_smem_set = 0;
    size_t grid_log[3] = {0, 0, 0};
    size_t grid_phy[3] = {0, 0, 0};
    size_t M = 0;
    double cell[6] = {4, 4, 4, 0, 0, 0};  // src/solver_base.h:43 default
    double ds = 0.0;
    bool ds_set = false;
    std::map<double, std::unique_ptr<OpsSet>> ops_cache;  // per ds, cleared by set_cell_para
    OpsSet* ops = nullptr;
    unsigned long long ops_gen = 0;  // bumped whenever `ops` may point elsewhere
    cudaStream_t stream = nullptr;      // where work is issued
    cudaStream_t own_stream = nullptr;  // created by the solver
    bool user_stream = false;
    double* iomat = nullptr;  // pinned host buffer (get_iomat_for_diffusion)
    DevBuf<double> d_io, d_t1, d_t2;
    size_t launches = 0;
    bool pmmm_anisotropic = false;  // PMMM with Lx, Ly, Lz (the reference's PMMM is cubic)
    M3Symmetry m3sym;                 // 3m mirror translations (decoded translational_part)
    std::vector<M3Term> m3terms;      // its Kronecker terms (one when the translations are 0)
    DevBuf<double> d_t3;              // input copy for in-place triplets of multi-term operators

    ~scft_solver_s() {
        if (iomat) cudaFreeHost(iomat);
        if (own_stream) cudaStreamDestroy(own_stream);
    }

    int nterms() const { return kind == SCFT_SOLVER_3M ? (int)m3terms.size() : 1; }
    bool m3_no_half_cells() const {
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
                if (m3sym.half[a][b]) return false;
        return true;
    }
    std::vector<const void*> fft_fn_set;  // FFT kernels granted their dynamic shared memory

    // whether the tensor-core axis passes (axis_dmma.cuh: FP64 DMMA; FP32: 3xTF32) run this
    // grid by default, on a cubic grid with a side the kernels cover (96 or 128), from
    // measurements on one B200: PMMM (two-level even/odd operators) always, 56 us against 65 us
    // by FFT per 256^3 triplet; P1 for both chains of an iteration (128^3: 52.5 against 49.4
    // iterations/s, precision form 69.7 against 62.1) but not for one chain (50 us by FFT
    // against 58 us); never 3m (128-point axes: 68 us by FFT against 82 us per triplet, 36.6
    // against 33.6 iterations/s at 256^3)
    template <typename T>
    bool tensor_axis_passes(int nchain) const {
        const OpsSet* o = ops;
        const int n = (int)grid_phy[0];
        if (kind == SCFT_SOLVER_3M || (kind == SCFT_SOLVER_P1 && nchain < 2)) return false;
        if (o->nterms != 1 || grid_phy[1] != grid_phy[0] || grid_phy[2] != grid_phy[0]) return false;
        size_t smem = 0, stride = 0;
        if constexpr (sizeof(T) == 8) {
            if (o->eo[0] != o->eo[1] || o->eo[1] != o->eo[2]) return false;
            return axis_dmma_kernel_for(n, o->eo[0], 2, &smem, o->eo2 && n == 128) != nullptr;
        } else {
            if (o->eo_f32[0] != o->eo_f32[1] || o->eo_f32[1] != o->eo_f32[2]) return false;
            return axis_tf32_kernel_for(n, o->eo_f32[0], 2, &smem, &stride) != nullptr;
        }
    }

    // the three passes of a triplet by FFT (axis_fft.cuh); *done = false if an axis has no
    // FFT form or the dense form is to run
    template <typename T>
    int triplet_fft(int nchain, const ChainIO<T> io[2], T* t1[2], T* t2[2], cudaStream_t st, bool* done) {
        *done = false;
        const OpsSet* o = ops;
        if (o->nterms != 1) return SCFT_OK;
        const int form = axis_form_override();
        if (form == 2) return SCFT_OK;
        if (form == 0 && tensor_axis_passes<T>(nchain)) return SCFT_OK;  // measured faster there
        AxisFftFn<T> f[3];
        size_t sm[3];
        for (int ax = 0; ax < 3; ++ax) {
            if (!o->fft_nf[ax]) return SCFT_OK;
            f[ax] = axis_fft_kernel_for<T>((int)grid_phy[ax], o->fft_nf[ax], o->fft_ext[ax], &sm[ax]);
            if (!f[ax]) return SCFT_OK;
        }
        if (!sms) CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        const int nx = (int)grid_phy[0], ny = (int)grid_phy[1], nz = (int)grid_phy[2];
        for (int ax = 2; ax >= 0; --ax) {
            bool set = false;
            for (const void* p : fft_fn_set) set |= p == (const void*)f[ax];
            if (!set) {
                CK(cudaFuncSetAttribute(f[ax], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm[ax]));
                fft_fn_set.push_back((const void*)f[ax]);
            }
            AxisFftPass<T> p{};
            for (int c = 0; c < nchain; ++c) {
                p.in[c] = ax == 2 ? io[c].in : (ax == 1 ? t1[c] : t2[c]);
                p.out[c] = ax == 2 ? t1[c] : (ax == 1 ? t2[c] : io[c].out);
                p.pre[c] = ax == 2 ? io[c].pre : nullptr;
                p.post[c] = ax == 0 ? io[c].post : nullptr;
            }
            p.nchain = nchain;
            if constexpr (sizeof(T) == 8) {
                p.tw = o->d_fft_tw[ax].p;
                p.g = o->d_fft_g[ax].p;
            } else {
                p.tw = o->f_fft_tw[ax].p;
                p.g = o->f_fft_g[ax].p;
            }
            p.outer = ax == 2 ? (long long)nx * ny : (ax == 1 ? nx : 1);
            p.inner = ax == 2 ? 1 : (ax == 1 ? nz : (long long)ny * nz);
            int per_sm = 1;
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f[ax], kFftThreads, sm[ax]));
            f[ax]<<<sms * (per_sm > 0 ? per_sm : 1), kFftThreads, sm[ax], st>>>(p);
            CK(cudaGetLastError());
        }
        launches += 3;
        *done = true;
        return SCFT_OK;
    }

    int build_ops(double ds_) {
        auto s = std::make_unique<OpsSet>();
        const int nt = nterms();
        s->nterms = nt;
        for (int t = 1; t < nt; ++t) s->more.push_back(std::make_unique<OpsSet>());
        int eo2_axes = 0;
        for (int ax = 0; ax < 3; ++ax) {
            std::vector<long double> A;
            const int N = (int)grid_log[ax];
            if (kind == SCFT_SOLVER_PMMM) {
                A = pmmm_axis_operator(N / 2, (long double)cell[ax], (long double)ds_);
            } else if (kind == SCFT_SOLVER_P1) {
                A = p1_axis_operator(N, (long double)cell[ax], (long double)ds_);
            } else {
                const std::vector<long double> c = circulant_kernel(N, (long double)cell[ax], (long double)ds_);
                for (int t = 1; t < nt; ++t)
                    CKR(upload_operator(m3_axis_factor(c, N, m3sym.par[ax], m3terms[(size_t)t][ax]),
                                        (int)grid_phy[ax], *s->term(t), ax));
                A = m3_axis_factor(c, N, m3sym.par[ax], m3terms[0][ax]);
            }
            CKR(upload_operator(A, (int)grid_phy[ax], *s, ax));
            pack_operator(A, (int)grid_phy[ax], *s, ax);
            pack_operator_f32(A, (int)grid_phy[ax], *s, ax);
            if (nt == 1 && s->h16_axes == ax) pack_operator_h16(A, (int)grid_phy[ax], *s);
            {
                const int n = (int)grid_phy[ax];
                int nf = 0, ext = 0;
                const bool m3_plain = kind == SCFT_SOLVER_3M && nt == 1 && m3sym.par[0] == 0 && m3sym.par[1] == 0 &&
                                      m3sym.par[2] == 0 && m3_no_half_cells();
                if (kind == SCFT_SOLVER_P1) nf = n;
                else if (kind == SCFT_SOLVER_PMMM) { nf = 2 * n; ext = 1; }
                else if (m3_plain) { nf = 2 * n; ext = 2; }
                size_t fsm = 0;
                if (nf && axis_fft_kernel_for<double>(n, nf, ext, &fsm))
                    CKR(upload_fft_tables(*s, ax, nf, ext, (long double)cell[ax], (long double)ds_));
            }
            eo2_axes += (kind == SCFT_SOLVER_PMMM && nt == 1 && pack_operator_eo2(A, (int)grid_phy[ax], *s)) ? 1 : 0;
        }
        s->eo2 = eo2_axes == 3;
        if (s->eo2) {
            CKR(s->d_packed2.alloc(s->h_packed2.size()));
            CKR(upload(s->d_packed2.p, s->h_packed2.data(), s->h_packed2.size() * sizeof(double)));
        }
        CKR(s->d_packed.alloc(s->h_packed.size()));
        CKR(upload(s->d_packed.p, s->h_packed.data(), s->h_packed.size() * sizeof(double)));
        CKR(s->f_packed.alloc(s->h_packed_f32.size()));
        CKR(upload(s->f_packed.p, s->h_packed_f32.data(), s->h_packed_f32.size() * sizeof(float)));
        if (s->h16_axes == 3) {
            CKR(s->h16_packed.alloc(s->h_packed_h16.size()));
            CKR(upload(s->h16_packed.p, s->h_packed_h16.data(), s->h_packed_h16.size() * sizeof(uint16_t)));
        }
        ops = s.get();
        ops_cache[ds_] = std::move(s);
        ++ops_gen;
        return SCFT_OK;
    }

    // the cell-length derivative operators of the current (cell, ds)
    int build_dops() {
        if (!ops) return fail(SCFT_ERR_NOT_READY, "set_cell_para/set_contour_step first");
        if (ops->have_dop) return SCFT_OK;
        for (int ax = 0; ax < 3; ++ax) {
            const int N = (int)grid_log[ax];
            const int n = (int)grid_phy[ax];
            std::vector<long double> dc;
            if (kind == SCFT_SOLVER_3M) dc = circulant_kernel_dL(N, (long double)cell[ax], (long double)ds);
            for (int t = 0; t < ops->nterms; ++t) {
                std::vector<long double> A;
                if (kind == SCFT_SOLVER_PMMM)
                    A = pmmm_axis_operator_dL(N / 2, (long double)cell[ax], (long double)ds);
                else if (kind == SCFT_SOLVER_P1)
                    A = p1_axis_operator_dL(N, (long double)cell[ax], (long double)ds);
                else
                    A = m3_axis_factor(dc, N, m3sym.par[ax], m3terms[(size_t)t][ax]);
                std::vector<double> d((size_t)n * n), dt((size_t)n * n);
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < n; ++j) {
                        d[(size_t)i * n + j] = (double)A[(size_t)i * n + j];
                        dt[(size_t)j * n + i] = (double)A[(size_t)i * n + j];
                    }
                OpsSet* o = ops->term(t);
                CKR(o->d_dop[ax].alloc((size_t)n * n));
                CKR(o->d_dopT[ax].alloc((size_t)n * n));
                CKR(upload(o->d_dop[ax].p, d.data(), d.size() * sizeof(double)));
                CKR(upload(o->d_dopT[ax].p, dt.data(), dt.size() * sizeof(double)));
            }
        }
        ops->have_dop = true;
        return SCFT_OK;
    }

    // (op_x (x) op_y (x) op_z) applied to nt stacked fields: in -> t1 -> t2 -> out
    int triplet_batched(const double* in, double* out, double* t1, double* t2, long long nt,
                        const double* const op[3], const double* const opT[3], cudaStream_t st) {
        const int nx = (int)grid_phy[0], ny = (int)grid_phy[1], nz = (int)grid_phy[2];
        AxisPass<double> pz{}, py{}, px{};
        pz.ch[0] = ChainIO<double>{in, t1, nullptr, nullptr};
        py.ch[0] = ChainIO<double>{t1, t2, nullptr, nullptr};
        px.ch[0] = ChainIO<double>{t2, out, nullptr, nullptr};
        pz.op = op[2]; pz.opT = opT[2]; pz.n = nz; pz.outer = nt * nx * ny; pz.inner = 1;
        py.op = op[1]; py.opT = opT[1]; py.n = ny; py.outer = nt * nx; py.inner = nz;
        px.op = op[0]; px.opT = opT[0]; px.n = nx; px.outer = nt; px.inner = (long long)ny * nz;
        CK(launch_axis(pz, 1, true, st));
        CK(launch_axis(py, 1, false, st));
        CK(launch_axis(px, 1, false, st));
        return SCFT_OK;
    }

    // one triplet per chain: in -> (pre) z-pass -> t1 -> y-pass -> t2 -> x-pass (post) -> out
    // A multi-term operator (ops->nterms > 1) runs the three passes per term and adds the
    // x passes up in `out`, so there `in` and `out` must not alias.
    template <typename T>
    int triplet(int nchain, const ChainIO<T> io[2], T* t1[2], T* t2[2], cudaStream_t st) {
        const int nx = (int)grid_phy[0], ny = (int)grid_phy[1], nz = (int)grid_phy[2];
        const int nt = ops->nterms;
        for (int c = 0; c < nchain && nt > 1; ++c)
            if ((const void*)io[c].in == (const void*)io[c].out)
                return fail(SCFT_ERR_INVALID_ARG, "multi-term triplet: input and output alias");
        {
            bool done = false;
            CKR(triplet_fft<T>(nchain, io, t1, t2, st, &done));
            if (done) return SCFT_OK;
        }
        if constexpr (sizeof(T) == 8) {
            // large cubic grids: the three passes on the FP64 tensor cores (axis_dmma.cuh)
            if (nt == 1 && nx == ny && ny == nz && ops->eo[0] == ops->eo[1] && ops->eo[1] == ops->eo[2]) {
                AxisDmmaFn f[3];
                size_t smem = 0;
                const bool eo2 = ops->eo2 && nx == 128;
                for (int ax = 0; ax < 3; ++ax) f[ax] = axis_dmma_kernel_for(nx, ops->eo[ax], ax, &smem, eo2);
                if (f[0] && f[1] && f[2]) {
                    if (!sms) CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
                    if (axis_dmma_smem_set != smem || axis_dmma_fn_set != (const void*)f[2]) {
                        for (int ax = 0; ax < 3; ++ax)
                            CK(cudaFuncSetAttribute(f[ax], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                        axis_dmma_smem_set = smem;
                        axis_dmma_fn_set = (const void*)f[2];
                    }
                    AxisPassD pz{}, py{}, px{};
                    for (int c = 0; c < nchain; ++c) {
                        pz.in[c] = io[c].in; pz.out[c] = t1[c]; pz.pre[c] = io[c].pre;
                        py.in[c] = t1[c]; py.out[c] = t2[c];
                        px.in[c] = t2[c]; px.out[c] = io[c].out; px.post[c] = io[c].post;
                    }
                    pz.nchain = py.nchain = px.nchain = nchain;
                    pz.hints = py.hints = px.hints = l2_hints_enabled();
                    py.discard_in = px.discard_in = l2_hints_enabled();  // t1, t2: dead once read
                    if (eo2) {
                        const size_t per_axis = ops->h_packed2.size() / 3;  // AxisShapeEO2<n>::SIZE
                        pz.op = ops->d_packed2.p + 2 * per_axis;
                        py.op = ops->d_packed2.p + per_axis;
                        px.op = ops->d_packed2.p;
                    } else {
                        pz.op = ops->d_packed.p + ops->off[2];
                        py.op = ops->d_packed.p + ops->off[1];
                        px.op = ops->d_packed.p + ops->off[0];
                    }
                    f[2]<<<sms, kContourThreads, smem, st>>>(pz);
                    CK(cudaGetLastError());
                    f[1]<<<sms, kContourThreads, smem, st>>>(py);
                    CK(cudaGetLastError());
                    f[0]<<<sms, kContourThreads, smem, st>>>(px);
                    CK(cudaGetLastError());
                    launches += 3;
                    return SCFT_OK;
                }
            }
        } else {
            // large cubic grids, FP32 precision form: 3xTF32 axis passes
            if (nt == 1 && nx == ny && ny == nz && ops->eo_f32[0] == ops->eo_f32[1] &&
                ops->eo_f32[1] == ops->eo_f32[2]) {
                AxisTf32Fn f[3];
                size_t smem = 0, stride = 0;
                for (int ax = 0; ax < 3; ++ax) f[ax] = axis_tf32_kernel_for(nx, ops->eo_f32[ax], ax, &smem, &stride);
                if (f[0] && f[1] && f[2]) {
                    if (!sms) CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
                    if (axis_tf32_smem_set != smem) {
                        for (int ax = 0; ax < 3; ++ax)
                            CK(cudaFuncSetAttribute(f[ax], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                        axis_tf32_smem_set = smem;
                    }
                    int per_sm = 1;
                    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f[2], kContourThreads, smem));
                    const int grid = sms * (per_sm > 0 ? per_sm : 1);
                    AxisPassF pz{}, py{}, px{};
                    for (int c = 0; c < nchain; ++c) {
                        pz.in[c] = (const float*)io[c].in; pz.out[c] = (float*)t1[c]; pz.pre[c] = (const float*)io[c].pre;
                        py.in[c] = (const float*)t1[c]; py.out[c] = (float*)t2[c];
                        px.in[c] = (const float*)t2[c]; px.out[c] = (float*)io[c].out;
                        px.post[c] = (const float*)io[c].post;
                    }
                    pz.nchain = py.nchain = px.nchain = nchain;
                    pz.hints = py.hints = px.hints = l2_hints_enabled();
                    py.discard_in = px.discard_in = l2_hints_enabled();  // t1, t2: dead once read
                    pz.op = ops->f_packed.p + 2 * stride;
                    py.op = ops->f_packed.p + stride;
                    px.op = ops->f_packed.p;
                    f[2]<<<grid, kContourThreads, smem, st>>>(pz);
                    CK(cudaGetLastError());
                    f[1]<<<grid, kContourThreads, smem, st>>>(py);
                    CK(cudaGetLastError());
                    f[0]<<<grid, kContourThreads, smem, st>>>(px);
                    CK(cudaGetLastError());
                    launches += 3;
                    return SCFT_OK;
                }
            }
        }
        for (int t = 0; t < nt; ++t) {
            OpsSet* o = ops->term(t);
            const T* opx;
            const T* opy;
            const T* opz;
            const T* opxT;
            const T* opyT;
            const T* opzT;
            if constexpr (sizeof(T) == 8) {
                opx = (const T*)o->d_op[0].p; opy = (const T*)o->d_op[1].p; opz = (const T*)o->d_op[2].p;
                opxT = (const T*)o->d_opT[0].p; opyT = (const T*)o->d_opT[1].p; opzT = (const T*)o->d_opT[2].p;
            } else {
                opx = (const T*)o->f_op[0].p; opy = (const T*)o->f_op[1].p; opz = (const T*)o->f_op[2].p;
                opxT = (const T*)o->f_opT[0].p; opyT = (const T*)o->f_opT[1].p; opzT = (const T*)o->f_opT[2].p;
            }
            AxisPass<T> pz{}, py{}, px{};
            for (int c = 0; c < nchain; ++c) {
                pz.ch[c] = ChainIO<T>{io[c].in, t1[c], io[c].pre, nullptr};
                py.ch[c] = ChainIO<T>{t1[c], t2[c], nullptr, nullptr};
                px.ch[c] = ChainIO<T>{t2[c], io[c].out, nullptr, t == nt - 1 ? io[c].post : nullptr, t > 0};
            }
            pz.op = opz; pz.opT = opzT; pz.n = nz; pz.outer = (long long)nx * ny; pz.inner = 1;
            py.op = opy; py.opT = opyT; py.n = ny; py.outer = nx; py.inner = nz;
            px.op = opx; px.opT = opxT; px.n = nx; px.outer = 1; px.inner = (long long)ny * nz;
            CK(launch_axis(pz, nchain, true, st));
            CK(launch_axis(py, nchain, false, st));
            CK(launch_axis(px, nchain, false, st));
            launches += 3;
        }
        return SCFT_OK;
    }
};

struct scft_diblock_s {
    scft_solver_t solver = nullptr;
    double fA = 0, ds = 0, xN = 0, acc = 0;
    size_t NsA = 0, NsB = 0, U = 0, M = 0;
    int precision = SCFT_FP64;
    bool fields_set = false;
    DevBuf<double> wA, wB, phiA, phiB, ksi, partials, hist;
    DevBuf<double> d_wAds, d_wBds, d_q, d_qc, d_t[4];
    DevBuf<float> f_wAds, f_wBds, f_q, f_qc, f_t[4];
    DevBuf<IterState> state;
    unsigned hist_cap = 1024;
    // mixing: history 0 = simple mixing with acc (calc_new_fields); > 0 = Anderson mixing
    int mix_history = 0;
    double mix_beta = 0.0;
    DevBuf<double> and_W, and_R, and_partials;  // ring of (history + 1) x 2M iterates / residuals
    DevBuf<AndersonState> and_state;
    std::vector<double> last_residuals;         // rms residual of each iteration of the last run
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    size_t launches_per_iter = 0;
    unsigned long long captured_gen = ~0ULL;
    cudaEvent_t* phase_events = nullptr;  // set by scft_diblock_time_phases (non-graph runs)
    bool use_graph = true;                // cleared if a capture is refused
    bool persistent = false;              // whole-contour cooperative kernel eligible
    int persistent_grid = 0;
    size_t persistent_smem = 0;
    ContourFn contour_fn = nullptr;
    bool alternating = false;             // contour_fn is the alternating-layout kernel
    bool alt_eo2 = false;                 // ... in its two-level even/odd form (operators d_packed2)
    int force_form = 0;                   // 0 auto, 1 alternating, 2 two-phase, 3 per-axis kernels
    int last_form = 0;                    // force_form the current launch plan was built with
    DevBuf<double> d_xch;                 // exchange buffers, 2 x space_size_phy per chain
    DevBuf<unsigned> flags;               // per-unit phase flags of the alternating kernel
    bool fused_phi = true;                // FP64 alternating kernel sums phi itself (scft_diblock_set_phi_form)
    bool phi_fused = false;               // the last launch_contour[_f32] ran with the fused phi sums
    bool f32_phi_fused = false;           // the FP32 launch plan has room for them (setup_persistent_f32)
    DevBuf<double> phi_acc;               // its sums: [chain][block][layout][tile][n^2], 8 x space_size_phy
    int last_iter_precision = -1;         // precision of the iteration whose contour is stored
    DevBuf<double> stress_buf;            // batched temporaries of scft_diblock_stress
    ContourFnF contour_fn_f32 = nullptr;  // FP32 (3xTF32) contour kernel
    bool cluster_f32 = false;             // FP32 runs on the cluster kernel (contour_cluster_f32.cuh)
    DevBuf<float> f_xch;                  // FP32 exchange buffers
    DevBuf<unsigned> ctrl;                // [0] barrier arrivals, [1] error bits
    long long spin_limit = 20000000LL;

    // graphs of the precision not in use (see scft_diblock_set_precision)
    cudaGraph_t saved_graph[2] = {nullptr, nullptr};
    cudaGraphExec_t saved_gexec[2] = {nullptr, nullptr};
    unsigned long long saved_gen[2] = {~0ULL, ~0ULL};
    bool saved_use_graph[2] = {true, true};

    // page-locked staging of the end-to-end form: hist_cap history rows, then the error word
    double* pin_out = nullptr;

    ~scft_diblock_s() {
        if (pin_out) cudaFreeHost(pin_out);
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        for (int i = 0; i < 2; ++i) {
            if (saved_gexec[i]) cudaGraphExecDestroy(saved_gexec[i]);
            if (saved_graph[i]) cudaGraphDestroy(saved_graph[i]);
        }
    }

    // Decide whether the persistent contour kernel can run this grid (FP64, every
    // axis a multiple of 8 and at most kContourMaxN, shared memory within the limit).
    // FP32 precision form: the 3xTF32 alternating kernel for cubic grids it covers
    // FP32 on clusters: 64^3 grids whose three axis operators are centrosymmetric (PMMM,
    // P1), when two 16-CTA clusters with the kernel's shared memory can be resident
    int setup_cluster_f32() {
        cluster_f32 = false;
        const OpsSet* o = solver->ops;
        if (!o || o->h16_axes != 3 || !o->h16_packed.p || force_form != 0) return SCFT_OK;
        const size_t* g = solver->grid_phy;
        if (g[0] != (size_t)kClN || g[1] != (size_t)kClN || g[2] != (size_t)kClN) return SCFT_OK;
        {
            const char* e = getenv("CRYSSCFT_FP32_CLUSTER");
            if (!e || e[0] != '1') return SCFT_OK;
        }
        int dev_smem = 0;
        CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, solver->device));
        if (kClSmem > (size_t)dev_smem) return SCFT_OK;
        CK(cudaFuncSetAttribute(contour_cluster_kernel_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClSmem));
        CK(cudaFuncSetAttribute(contour_cluster_kernel_f32, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[1];
        cluster_config(cfg, attr, nullptr);
        int nclusters = 0;
        if (cudaOccupancyMaxActiveClusters(&nclusters, contour_cluster_kernel_f32, &cfg) != cudaSuccess) {
            cudaGetLastError();
            return SCFT_OK;
        }
        if (nclusters < 2) return SCFT_OK;
        if (!ctrl.p) {
            CKR(ctrl.alloc(2));
            CKR(zero_device(ctrl.p, 2 * sizeof(unsigned)));
        }
        cluster_f32 = true;
        persistent = true;
        alternating = true;
        return SCFT_OK;
    }

    void cluster_config(cudaLaunchConfig_t& cfg, cudaLaunchAttribute* attr, cudaStream_t st) const {
        cfg.gridDim = dim3(2 * kClCtas);
        cfg.blockDim = dim3(kClThreads);
        cfg.dynamicSmemBytes = kClSmem;
        cfg.stream = st;
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kClCtas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }

    int launch_cluster_f32(cudaStream_t st, float* wAds, float* wBds, float* q, float* qc) {
        ClusterArgsF a{};
        a.q[0] = q;
        a.q[1] = qc;
        a.wds[0] = wAds;
        a.wds[1] = wBds;
        a.ops = solver->ops->h16_packed.p;
        a.slot0[0] = 0;
        a.dir[0] = 1;
        a.slot0[1] = (long long)U;
        a.dir[1] = -1;
        a.NsA = (long long)NsA;
        a.U = (int)U;
        a.error = reinterpret_cast<int*>(ctrl.p + 1);
        a.spin_limit = spin_limit;
        cudaLaunchConfig_t cfg{};
        cudaLaunchAttribute attr[1];
        cluster_config(cfg, attr, st);
        CK(cudaLaunchKernelEx(&cfg, contour_cluster_kernel_f32, a));
        return SCFT_OK;
    }

    int setup_persistent_f32() {
        persistent = false;
        f32_phi_fused = false;
        CKR(setup_cluster_f32());
        if (cluster_f32) return SCFT_OK;
        const OpsSet* o = solver->ops;
        if (!o) return SCFT_OK;
        const int nx = (int)solver->grid_phy[0], ny = (int)solver->grid_phy[1], nz = (int)solver->grid_phy[2];
        if (nx != ny || ny != nz || o->eo_f32[0] != o->eo_f32[1] || o->eo_f32[1] != o->eo_f32[2]) return SCFT_OK;
        size_t smem = 0;
        ContourFnF f = contour_alt_kernel_f32_for(nx, o->eo_f32[0], &smem);
        if (!f) return SCFT_OK;
        int dev_smem = 0, sms = 0;
        CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, solver->device));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, solver->device));
        if (smem > (size_t)dev_smem) return SCFT_OK;
        // fused phi sums: two more tiles (the other chain's FP32 tile, the FP64 products)
        // where they fit (AltShapeF::SMEM_FUSED)
        const size_t smem_fused = smem + (size_t)nx * nx * (sizeof(float) + sizeof(double));
        f32_phi_fused = fused_phi && U % 2 == 0 && NsA >= 1 && NsB >= 1 && smem_fused <= (size_t)dev_smem;
        if (f32_phi_fused) smem = smem_fused;
        CK(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kContourThreads, smem));
        if (per_sm < 1) return SCFT_OK;
        if (2 * nx > per_sm * sms) return SCFT_OK;  // one unit per block
        contour_fn_f32 = f;
        persistent_grid = 2 * nx;
        persistent_smem = smem;
        if (!f_xch.p) CKR(f_xch.alloc(4 * M));
        if (flags.n != alt_flag_count(nx)) CKR(flags.alloc(alt_flag_count(nx)));
        if (!ctrl.p) {
            CKR(ctrl.alloc(2));
            CKR(zero_device(ctrl.p, 2 * sizeof(unsigned)));
        }
        alternating = true;
        persistent = true;
        return SCFT_OK;
    }

    int launch_contour_f32(cudaStream_t st, float* wAds, float* wBds, float* q, float* qc) {
        phi_fused = false;
        if (cluster_f32) return launch_cluster_f32(st, wAds, wBds, q, qc);
        ContourArgsF a{};
        a.q[0] = q;
        a.q[1] = qc;
        a.wds[0] = wAds;
        a.wds[1] = wBds;
        a.xbuf[0] = f_xch.p;
        a.xbuf[1] = f_xch.p + 2 * M;
        a.ops = solver->ops->f_packed.p;
        a.nchain = 2;
        a.slot0[0] = 0;
        a.dir[0] = 1;
        a.slot0[1] = (long long)U;
        a.dir[1] = -1;
        a.NsA = (long long)NsA;
        a.t_end = (int)U;
        a.error = reinterpret_cast<int*>(ctrl.p + 1);
        a.spin_limit = spin_limit;
        a.flags = flags.p;
        const int n = (int)solver->grid_phy[0];
        phi_fused = f32_phi_fused;  // set up with the launch's shared memory size
        if (phi_fused) {
            if (phi_acc.n != 8 * M) CKR(phi_acc.alloc(8 * M));
            a.phi_acc = phi_acc.p;
            a.done = flags.p + 4 * (size_t)n * n;
        }
        for (int v = 0; v < 2; ++v) {  // panel tiles, plane [0] and slab [1] views
            CKR(encode_panel_map(&a.tm_pq[0][v], q, n, (long long)U + 1, v == 0, false));
            CKR(encode_panel_map(&a.tm_pq[1][v], qc, n, (long long)U + 1, v == 0, false));
            CKR(encode_panel_map(&a.tm_pw[0][v], wAds, n, 0, v == 0, false));
            CKR(encode_panel_map(&a.tm_pw[1][v], wBds, n, 0, v == 0, false));
        }
        CK(cudaMemsetAsync(flags.p, 0, flags.n * sizeof(unsigned), st));
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)persistent_grid);
        cfg.blockDim = dim3(kContourThreads);
        cfg.dynamicSmemBytes = persistent_smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, contour_fn_f32, a));
        return SCFT_OK;
    }

    int setup_persistent() {
        persistent = false;
        alternating = false;
        alt_eo2 = false;
        if (force_form == 3) return SCFT_OK;  // per-axis kernels only
        if (solver->ops && solver->ops->nterms > 1) return SCFT_OK;  // multi-term: per-axis kernels
        if (precision == SCFT_FP32) return setup_persistent_f32();
        const OpsSet* o = solver->ops;
        if (!o) return SCFT_OK;
        for (int ax = 0; ax < 3; ++ax) {
            const size_t n = solver->grid_phy[ax];
            if (n < 8 || n % 8 || n > (size_t)kContourMaxN) return SCFT_OK;
        }
        const int nx = (int)solver->grid_phy[0], ny = (int)solver->grid_phy[1], nz = (int)solver->grid_phy[2];
        const int rows = nx > ny ? nx : ny;
        size_t smem = ((size_t)((o->total + 1) & ~1) + 2 * (size_t)rows * (nz + 4)) * sizeof(double);
        int dev_smem = 0, sms = 0;
        CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, solver->device));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, solver->device));
        if (smem > (size_t)dev_smem) return SCFT_OK;
        contour_fn = contour_kernel_for(nx, ny, nz, o->eo);
        alternating = false;
        if (nx == ny && ny == nz && o->eo[0] == o->eo[1] && o->eo[1] == o->eo[2] && force_form != 2) {
            size_t alt_smem = 0;
            ContourFn f = contour_alt_kernel_for(nx, o->eo[0], &alt_smem, o->eo2);
            alt_eo2 = f && o->eo2 && nx == 64;
            if (f && alt_smem <= (size_t)dev_smem) {
                contour_fn = f;
                smem = alt_smem;
                alternating = true;
            } else {
                alt_eo2 = false;
            }
        }
        if (!d_xch.p) CKR(d_xch.alloc(4 * M));
        if (alternating && flags.n != alt_flag_count(nx)) CKR(flags.alloc(alt_flag_count(nx)));
        CK(cudaFuncSetAttribute(contour_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, contour_fn, kContourThreads, smem));
        if (per_sm < 1) return SCFT_OK;
        const int units = 2 * (nx > ny ? nx : ny);
        if (alternating && units > per_sm * sms) return SCFT_OK;  // one unit per block: per-axis kernels
        persistent_grid = std::min(units, per_sm * sms);
        persistent_smem = smem;
        if (!ctrl.p) {
            CKR(ctrl.alloc(2));
            CKR(zero_device(ctrl.p, 2 * sizeof(unsigned)));
        }
        persistent = true;
        return SCFT_OK;
    }

    int launch_contour(cudaStream_t st, double* wAds, double* wBds, double* q, double* qc) {
        const OpsSet* o = solver->ops;
        ContourArgs a{};
        a.q[0] = q;
        a.q[1] = qc;
        a.wds[0] = wAds;
        a.wds[1] = wBds;
        a.xbuf[0] = d_xch.p;          // 2M per chain: plane- and slab-phase exchange buffers
        a.xbuf[1] = d_xch.p + 2 * M;
        a.ops = alt_eo2 ? o->d_packed2.p : o->d_packed.p;
        for (int ax = 0; ax < 3; ++ax) {
            a.n[ax] = (int)solver->grid_phy[ax];
            a.eo[ax] = o->eo[ax];
            a.op_off[ax] = o->off[ax];
            a.op_ld[ax] = o->ld[ax];
            a.op_half[ax] = o->half[ax];
        }
        a.ops_total = o->total;
        a.nchain = 2;
        a.slot0[0] = 0;
        a.dir[0] = 1;
        a.slot0[1] = (long long)U;
        a.dir[1] = -1;
        a.NsA = (long long)NsA;
        a.t_begin = 0;
        a.t_end = (int)U;
        a.bar_count = ctrl.p;
        a.error = reinterpret_cast<int*>(ctrl.p + 1);
        a.spin_limit = spin_limit;
        a.flags = flags.p;
        CK(cudaMemsetAsync(ctrl.p, 0, sizeof(unsigned), st));
        // phi summed inside the alternating kernel: both chains, U even (the slots the two
        // chains finish meet on the same layout), both blocks non-empty
        phi_fused = alternating && fused_phi && U % 2 == 0 && NsA >= 1 && NsB >= 1;
        if (phi_fused) {
            if (phi_acc.n != 8 * M) CKR(phi_acc.alloc(8 * M));
            a.phi_acc = phi_acc.p;
            a.done = flags.p + 4 * solver->grid_phy[0] * solver->grid_phy[0];
        }
        if (alternating) {
            const int n = (int)solver->grid_phy[0];
            for (int v = 0; v < 2; ++v) {  // panel tiles, plane [0] and slab [1] views
                CKR(encode_panel_map(&a.tm_pq[0][v], q, n, (long long)U + 1, v == 0));
                CKR(encode_panel_map(&a.tm_pq[1][v], qc, n, (long long)U + 1, v == 0));
                CKR(encode_panel_map(&a.tm_pw[0][v], wAds, n, 0, v == 0));
                CKR(encode_panel_map(&a.tm_pw[1][v], wBds, n, 0, v == 0));
            }
            CK(cudaMemsetAsync(flags.p, 0, flags.n * sizeof(unsigned), st));
        }
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)persistent_grid);
        cfg.blockDim = dim3(kContourThreads);
        cfg.dynamicSmemBytes = persistent_smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, contour_fn, a));
        return SCFT_OK;
    }

    // Parts of one iteration (bit mask): the batch kernel runs the contours of many
    // instances in one launch between the instances' prep and field parts.
    static constexpr int kPartPrep = 1, kPartContour = 2, kPartFields = 4, kPartAll = 7;

    template <typename T>
    int enqueue_iteration(cudaStream_t st, T* wAds, T* wBds, T* q, T* qc, T** t, int parts = kPartAll) {
        const long long MM = (long long)M;
        const int blocks = grid_blocks(MM, 256);
        size_t launches = 0;
        bool fused = false;  // phi was summed by this iteration's contour kernel
        if (parts & kPartPrep) {
            prep_kernel<T><<<blocks, 256, 0, st>>>(wA.p, wB.p, ksi.p, wAds, wBds, q, qc + U * M, xN, ds, MM);
            CK(cudaGetLastError());
            ++launches;
        }
        if (parts & kPartContour) {
            if (phase_events) CK(cudaEventRecord(phase_events[1], st));
            const size_t before = solver->launches;
            if (persistent) {
                if constexpr (sizeof(T) == 8) {
                    CKR(launch_contour(st, wAds, wBds, q, qc));
                    fused = phi_fused;
                } else {
                    CKR(launch_contour_f32(st, wAds, wBds, q, qc));
                    fused = phi_fused;
                }
                ++solver->launches;
            }
            for (size_t t_ = 0; t_ < U && !persistent; ++t_) {
                // forward chain: q[t] -> q[t+1] with block A (t < NsA) or B
                // backward chain: qc[U-t] -> qc[U-t-1] with the block of segment U-t-1
                const T* w1 = t_ < NsA ? wAds : wBds;
                const size_t ub = U - t_ - 1;
                const T* w2 = ub < NsA ? wAds : wBds;
                ChainIO<T> io[2];
                io[0] = ChainIO<T>{q + t_ * M, q + (t_ + 1) * M, w1, w1};
                io[1] = ChainIO<T>{qc + (ub + 1) * M, qc + ub * M, w2, w2};
                T* t1[2] = {t[0], t[1]};
                T* t2[2] = {t[2], t[3]};
                CKR(solver->triplet<T>(2, io, t1, t2, st));
            }
            launches += solver->launches - before;
            if (phase_events) CK(cudaEventRecord(phase_events[2], st));
        }
        if (!(parts & kPartFields)) {
            launches_per_iter = launches;
            return SCFT_OK;
        }
        const int rblocks = (int)std::min<long long>(kRedMaxBlocks, (MM + kRedThreads - 1) / kRedThreads);
        q_reduce_kernel<T><<<rblocks, kRedThreads, 0, st>>>(qc, MM, partials.p, state.p);
        CK(cudaGetLastError());
        if (fused)
            phi_fused_finish_kernel<T><<<grid_blocks(MM, 256), 256, 0, st>>>(
                phi_acc.p, q, qc, phiA.p, phiB.p, state.p, fA, (long long)NsA, (long long)NsB,
                (int)solver->grid_phy[0]);
        else
            phi_kernel<T><<<grid_blocks((MM + 1) / 2, 256), 256, 0, st>>>(q, qc, phiA.p, phiB.p, state.p, fA,
                                                                          (long long)NsA, (long long)NsB, MM);
        CK(cudaGetLastError());
        if (phase_events) CK(cudaEventRecord(phase_events[3], st));
        energy_kernel<<<rblocks, kRedThreads, 0, st>>>(wA.p, wB.p, phiA.p, phiB.p, ksi.p, xN, MM,
                                                       partials.p, state.p, hist.p, hist_cap);
        CK(cudaGetLastError());
        if (mix_history > 0) {
            anderson_record_kernel<<<blocks, 256, 0, st>>>(wA.p, wB.p, phiA.p, phiB.p, ksi.p, xN, MM, and_W.p,
                                                          and_R.p, and_state.p);
            CK(cudaGetLastError());
            const int dblocks = (int)std::min<long long>(kRedMaxBlocks, (2 * MM + kRedThreads - 1) / kRedThreads);
            anderson_dots_kernel<<<dblocks, kRedThreads, 0, st>>>(and_R.p, MM, mix_history + 1, and_partials.p,
                                                                  and_state.p);
            CK(cudaGetLastError());
            anderson_solve_kernel<<<1, 32, 0, st>>>(and_state.p, mix_history);
            CK(cudaGetLastError());
            anderson_update_kernel<<<grid_blocks(2 * MM, 256), 256, 0, st>>>(wA.p, wB.p, and_W.p, and_R.p, MM,
                                                                          and_state.p, mix_beta, state.p);
            CK(cudaGetLastError());
            launches += 3 + 4;
        } else {
            update_kernel<<<blocks, 256, 0, st>>>(wA.p, wB.p, phiA.p, phiB.p, ksi.p, xN, acc, MM, state.p);
            CK(cudaGetLastError());
            launches += 4;
        }
        launches_per_iter = launches;
        return SCFT_OK;
    }

    int enqueue(cudaStream_t st, int parts = kPartAll) {
        if (precision == SCFT_FP64) {
            double* t[4] = {d_t[0].p, d_t[1].p, d_t[2].p, d_t[3].p};
            return enqueue_iteration<double>(st, d_wAds.p, d_wBds.p, d_q.p, d_qc.p, t, parts);
        }
        float* t[4] = {f_t[0].p, f_t[1].p, f_t[2].p, f_t[3].p};
        return enqueue_iteration<float>(st, f_wAds.p, f_wBds.p, f_q.p, f_qc.p, t, parts);
    }

    int ensure_graph() {
        if (gexec || !use_graph) return SCFT_OK;
        // capture on the solver's own (non-blocking) stream; the graph is launched on solver->stream
        cudaStream_t st = solver->own_stream;
        CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        int r = enqueue(st);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &g);
        if (r != SCFT_OK || e != cudaSuccess) {
            // capture refused (e.g. a launch form the runtime cannot record): run uncaptured
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            use_graph = false;
            return SCFT_OK;
        }
        graph = g;
        if (cudaGraphInstantiate(&gexec, graph, 0) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphDestroy(graph);
            graph = nullptr;
            gexec = nullptr;
            use_graph = false;
        }
        return SCFT_OK;
    }

    int run_once(cudaStream_t st) {
        if (gexec) {
            CK(cudaGraphLaunch(gexec, st));
            return SCFT_OK;
        }
        return enqueue(st);
    }
};

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* scft_last_error(void) { return g_last_error.c_str(); }

const char* scft_status_string(int s) {
    switch (s) {
        case SCFT_OK: return "SCFT_OK";
        case SCFT_ERR_INVALID_ARG: return "SCFT_ERR_INVALID_ARG";
        case SCFT_ERR_BAD_GRID: return "SCFT_ERR_BAD_GRID";
        case SCFT_ERR_CUDA: return "SCFT_ERR_CUDA";
        case SCFT_ERR_ALLOC: return "SCFT_ERR_ALLOC";
        case SCFT_ERR_NOT_READY: return "SCFT_ERR_NOT_READY";
        case SCFT_ERR_NUMERIC: return "SCFT_ERR_NUMERIC";
        case SCFT_ERR_TIMEOUT: return "SCFT_ERR_TIMEOUT";
        case SCFT_ERR_UNSUPPORTED: return "SCFT_ERR_UNSUPPORTED";
        case SCFT_ERR_NO_DEVICE: return "SCFT_ERR_NO_DEVICE";
        default: return "SCFT_ERR_UNKNOWN";
    }
}

const char* scft_version(void) { return "crysscft_b200 0.1 (sm_100a)"; }

int scft_solver_create(int kind, const size_t grid_size_log[3], const double translational_part[9],
                       int precision, int device, scft_solver_t* out) {
    if (!out || !grid_size_log) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (kind < SCFT_SOLVER_P1 || kind > SCFT_SOLVER_PMMM) return fail(SCFT_ERR_INVALID_ARG, "bad solver kind");
    if (precision != SCFT_FP64 && precision != SCFT_FP32) return fail(SCFT_ERR_INVALID_ARG, "bad precision");
    const size_t Nx = grid_size_log[0], Ny = grid_size_log[1], Nz = grid_size_log[2];
    // grid checks of the reference constructors (src/solver_p1.h:101-108,
    // src/solver_3m.h:81-92, src/solver_Pmmm.h:71-82); the GPU path has no alignment rule
    if (Nx == 0 || Ny == 0 || Nz == 0) return fail(SCFT_ERR_BAD_GRID, "ERROR: Bad Grid Size");
    if (kind != SCFT_SOLVER_P1 && (Nx % 2 || Ny % 2 || Nz % 2))
        return fail(SCFT_ERR_BAD_GRID, "ERROR: Grid Size Must Be Even For this symmetry");
    const size_t maxn = 1024;
    if (Nx > maxn || Ny > maxn || Nz > maxn) return fail(SCFT_ERR_BAD_GRID, "grid too large");
    M3Symmetry sym;
    if (kind == SCFT_SOLVER_3M && translational_part) {
        std::string why;
        if (!m3_symmetry_from_g(translational_part, grid_size_log, &sym, &why))
            return fail(SCFT_ERR_INVALID_ARG, "3m solver: " + why);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(SCFT_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0) CK(cudaGetDevice(&device));
    if (device >= ndev) return fail(SCFT_ERR_INVALID_ARG, "bad device ordinal");
    CK(cudaSetDevice(device));
    auto s = std::make_unique<scft_solver_s>();
    s->kind = kind;
    s->precision = precision;
    s->device = device;
    for (int i = 0; i < 3; ++i) {
        s->grid_log[i] = grid_size_log[i];
        s->grid_phy[i] = kind == SCFT_SOLVER_P1 ? grid_size_log[i] : grid_size_log[i] / 2;
    }
    s->M = s->grid_phy[0] * s->grid_phy[1] * s->grid_phy[2];
    if (kind == SCFT_SOLVER_3M) {
        s->m3sym = sym;
        s->m3terms = m3_terms(sym);
    }
    CK(cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking));
    s->stream = s->own_stream;
    cudaError_t e = cudaHostAlloc((void**)&s->iomat, s->M * sizeof(double), cudaHostAllocDefault);
    if (e != cudaSuccess) return fail(SCFT_ERR_ALLOC, "cudaHostAlloc iomat");
    std::memset(s->iomat, 0, s->M * sizeof(double));
    *out = s.release();
    return SCFT_OK;
}

int scft_operator_terms(int kind, const size_t grid_size_log[3], const double translational_part[9],
                        const double cell[3], double ds, size_t* nterms, double* factors, size_t capacity) {
    if (!grid_size_log || !cell || !nterms) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    if (kind < SCFT_SOLVER_P1 || kind > SCFT_SOLVER_PMMM) return fail(SCFT_ERR_INVALID_ARG, "bad solver kind");
    size_t N[3], n[3];
    for (int a = 0; a < 3; ++a) {
        N[a] = grid_size_log[a];
        if (N[a] == 0 || N[a] > 1024) return fail(SCFT_ERR_BAD_GRID, "ERROR: Bad Grid Size");
        if (kind != SCFT_SOLVER_P1 && N[a] % 2) return fail(SCFT_ERR_BAD_GRID, "ERROR: Grid Size Must Be Even");
        if (!(cell[a] > 0.0)) return fail(SCFT_ERR_INVALID_ARG, "cell lengths must be > 0");
        n[a] = kind == SCFT_SOLVER_P1 ? N[a] : N[a] / 2;
    }
    if (!(ds > 0.0)) return fail(SCFT_ERR_INVALID_ARG, "ds must be > 0");
    std::vector<M3Term> terms(1);
    M3Symmetry sym;
    if (kind == SCFT_SOLVER_3M) {
        if (translational_part) {
            std::string why;
            if (!m3_symmetry_from_g(translational_part, N, &sym, &why)) return fail(SCFT_ERR_INVALID_ARG, "3m solver: " + why);
        }
        terms = m3_terms(sym);
    }
    *nterms = terms.size();
    if (!factors) return SCFT_OK;
    const size_t need = terms.size() * (n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (capacity < need) return fail(SCFT_ERR_INVALID_ARG, "factors: capacity too small");
    double* o = factors;
    for (size_t t = 0; t < terms.size(); ++t)
        for (int a = 0; a < 3; ++a) {
            std::vector<long double> A;
            const long double L = (long double)cell[a], h = (long double)ds;
            if (kind == SCFT_SOLVER_PMMM) A = pmmm_axis_operator((int)n[a], L, h);
            else if (kind == SCFT_SOLVER_P1) A = p1_axis_operator((int)N[a], L, h);
            else A = m3_axis_factor(circulant_kernel((int)N[a], L, h), (int)N[a], sym.par[a], terms[t][a]);
            for (size_t i = 0; i < A.size(); ++i) *o++ = (double)A[i];
        }
    return SCFT_OK;
}

int scft_solver_destroy(scft_solver_t s) {
    if (!s) return SCFT_OK;
    if (s->users > 0) {  // iteration contexts still use it: freed with the last of them
        s->destroy_pending = true;
        return SCFT_OK;
    }
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    delete s;
    return SCFT_OK;
}

int scft_solver_set_pmmm_anisotropic(scft_solver_t s, int enable) {
    if (!s) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (s->kind != SCFT_SOLVER_PMMM) return fail(SCFT_ERR_INVALID_ARG, "only the PMMM solver has a cubic restriction");
    s->pmmm_anisotropic = enable != 0;
    // takes effect at the next set_cell_para (the cell in use is kept as it is)
    return SCFT_OK;
}

int scft_solver_set_cell_para(scft_solver_t s, const double c[6]) {
    if (!s || !c) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    for (int i = 0; i < 3; ++i)
        if (!(c[i] > 0.0) || !std::isfinite(c[i])) return fail(SCFT_ERR_INVALID_ARG, "cell lengths must be > 0");
    if (s->kind == SCFT_SOLVER_PMMM && !s->pmmm_anisotropic) {
        // src/solver_Pmmm.h:98-104: cubic, only cell_para[0] is used
        const double c6[6] = {c[0], c[0], c[0], 0, 0, 0};
        std::memcpy(s->cell, c6, sizeof(c6));
    } else {
        const double c6[6] = {c[0], c[1], c[2], 0, 0, 0};
        std::memcpy(s->cell, c6, sizeof(c6));
    }
    CK(cudaSetDevice(s->device));
    CK(cudaStreamSynchronize(s->stream));
    s->ops_cache.clear();
    s->ops = nullptr;
    ++s->ops_gen;
    s->ds = 0.0;
    s->ds_set = false;
    return SCFT_OK;
}

int scft_solver_set_contour_step(scft_solver_t s, double ds) {
    if (!s) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (!(ds > 0.0) || !std::isfinite(ds)) return fail(SCFT_ERR_INVALID_ARG, "ds must be > 0");
    CK(cudaSetDevice(s->device));
    s->ds = ds;
    s->ds_set = true;
    auto it = s->ops_cache.find(ds);
    if (it != s->ops_cache.end()) {
        if (s->ops != it->second.get()) ++s->ops_gen;
        s->ops = it->second.get();
        return SCFT_OK;
    }
    return s->build_ops(ds);
}

int scft_solver_get_grid_size_log(scft_solver_t s, size_t out[3]) {
    if (!s || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    for (int i = 0; i < 3; ++i) out[i] = s->grid_log[i];
    return SCFT_OK;
}
int scft_solver_get_grid_size_phy(scft_solver_t s, size_t out[3]) {
    if (!s || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    for (int i = 0; i < 3; ++i) out[i] = s->grid_phy[i];
    return SCFT_OK;
}
int scft_solver_get_space_size_phy(scft_solver_t s, size_t* out) {
    if (!s || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = s->M;
    return SCFT_OK;
}
int scft_solver_get_cell_para(scft_solver_t s, double out[6]) {
    if (!s || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    std::memcpy(out, s->cell, sizeof(s->cell));
    return SCFT_OK;
}
int scft_solver_get_ds(scft_solver_t s, double* out) {
    if (!s || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = s->ds;
    return SCFT_OK;
}
int scft_solver_get_iomat_for_diffusion(scft_solver_t s, double** out) {
    if (!s || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = s->iomat;
    return SCFT_OK;
}

static int solver_ready(scft_solver_t s) {
    if (!s) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (!s->ds_set || !s->ops) return fail(SCFT_ERR_NOT_READY, "set_cell_para/set_contour_step first");
    return SCFT_OK;
}

static int ensure_work(scft_solver_t s) {
    if (s->d_t1.n != s->M) {
        CKR(s->d_io.alloc(s->M));
        CKR(s->d_t1.alloc(s->M));
        CKR(s->d_t2.alloc(s->M));
    }
    if (s->nterms() > 1 && s->d_t3.n != s->M) CKR(s->d_t3.alloc(s->M));
    return SCFT_OK;
}

int scft_solver_diffusion_device(scft_solver_t s, double* d_io, void* stream) {
    CKR(solver_ready(s));
    if (!d_io) return fail(SCFT_ERR_INVALID_ARG, "null buffer");
    CK(cudaSetDevice(s->device));
    CKR(ensure_work(s));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    ChainIO<double> io[2] = {{d_io, d_io, nullptr, nullptr}, {}};
    // the z pass reads d_io into t1, the x pass writes d_io from t2: no aliasing inside a pass;
    // a multi-term operator reads its input once per term, so it works from a copy
    if (s->ops->nterms > 1) {
        CK(cudaMemcpyAsync(s->d_t3.p, d_io, s->M * sizeof(double), cudaMemcpyDeviceToDevice, st));
        io[0].in = s->d_t3.p;
    }
    double* t1[2] = {s->d_t1.p, nullptr};
    double* t2[2] = {s->d_t2.p, nullptr};
    return s->triplet<double>(1, io, t1, t2, st);
}

int scft_solver_diffusion(scft_solver_t s) {
    CKR(solver_ready(s));
    CK(cudaSetDevice(s->device));
    CKR(ensure_work(s));
    const size_t bytes = s->M * sizeof(double);
    CK(cudaMemcpyAsync(s->d_io.p, s->iomat, bytes, cudaMemcpyHostToDevice, s->stream));
    CKR(scft_solver_diffusion_device(s, s->d_io.p, s->stream));
    CK(cudaMemcpyAsync(s->iomat, s->d_io.p, bytes, cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCFT_OK;
}

int scft_solver_propagate_device(scft_solver_t s, double* d_q, const double* d_init,
                                 const double* d_wds, size_t Ns, int direction, void* stream) {
    CKR(solver_ready(s));
    if (!d_q || !d_init || !d_wds) return fail(SCFT_ERR_INVALID_ARG, "null buffer");
    if (direction != 1 && direction != -1) return fail(SCFT_ERR_INVALID_ARG, "Wrong direction");
    CK(cudaSetDevice(s->device));
    CKR(ensure_work(s));
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    const size_t M = s->M;
    size_t slot = direction == 1 ? 0 : Ns;
    CK(cudaMemcpyAsync(d_q + slot * M, d_init, M * sizeof(double), cudaMemcpyDeviceToDevice, st));
    for (size_t k = 0; k < Ns; ++k) {
        const size_t next = direction == 1 ? slot + 1 : slot - 1;
        ChainIO<double> io[2] = {{d_q + slot * M, d_q + next * M, d_wds, d_wds}, {}};
        double* t1[2] = {s->d_t1.p, nullptr};
        double* t2[2] = {s->d_t2.p, nullptr};
        CKR(s->triplet<double>(1, io, t1, t2, st));
        slot = next;
    }
    return SCFT_OK;
}

int scft_solver_propagate(scft_solver_t s, double* q, const double* init, const double* wds, size_t Ns,
                          int direction) {
    CKR(solver_ready(s));
    if (!q || !init || !wds) return fail(SCFT_ERR_INVALID_ARG, "null buffer");
    CK(cudaSetDevice(s->device));
    const size_t M = s->M;
    DevBuf<double> dq, di, dw;
    CKR(dq.alloc((Ns + 1) * M));
    CKR(di.alloc(M));
    CKR(dw.alloc(M));
    CK(cudaMemcpyAsync(di.p, init, M * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CK(cudaMemcpyAsync(dw.p, wds, M * sizeof(double), cudaMemcpyHostToDevice, s->stream));
    CKR(scft_solver_propagate_device(s, dq.p, di.p, dw.p, Ns, direction, s->stream));
    CK(cudaMemcpyAsync(q, dq.p, (Ns + 1) * M * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    CK(cudaStreamSynchronize(s->stream));
    return SCFT_OK;
}

// ------------------------------- diblock ----------------------------------
// Contour stores and Boltzmann factors of one precision (allocated on first use).
static int diblock_buffers(scft_diblock_t d, int precision) {
    const size_t M = d->M;
    if (precision == SCFT_FP64) {
        if (d->d_q.p) return SCFT_OK;
        CKR(d->d_wAds.alloc(M)); CKR(d->d_wBds.alloc(M));
        CKR(d->d_q.alloc((d->U + 1) * M)); CKR(d->d_qc.alloc((d->U + 1) * M));
        for (int i = 0; i < 4; ++i) CKR(d->d_t[i].alloc(M));
    } else {
        if (d->f_q.p) return SCFT_OK;
        CKR(d->f_wAds.alloc(M)); CKR(d->f_wBds.alloc(M));
        CKR(d->f_q.alloc((d->U + 1) * M)); CKR(d->f_qc.alloc((d->U + 1) * M));
        for (int i = 0; i < 4; ++i) CKR(d->f_t[i].alloc(M));
    }
    return SCFT_OK;
}

int scft_diblock_set_precision(scft_diblock_t d, int precision) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (precision != SCFT_FP64 && precision != SCFT_FP32) return fail(SCFT_ERR_INVALID_ARG, "bad precision");
    if (precision == d->precision) return SCFT_OK;
    CK(cudaSetDevice(d->solver->device));
    CK(cudaStreamSynchronize(d->solver->stream));
    CKR(diblock_buffers(d, precision));
    // keep the captured graph of each precision: switching back and forth (FP32 iterations,
    // then FP64 polish) replays instead of re-capturing
    const int o = d->precision, n = precision;
    d->saved_graph[o] = d->graph;
    d->saved_gexec[o] = d->gexec;
    d->saved_gen[o] = d->captured_gen;
    d->saved_use_graph[o] = d->use_graph;
    d->graph = d->saved_graph[n];
    d->gexec = d->saved_gexec[n];
    d->captured_gen = d->saved_gen[n];
    d->use_graph = d->saved_use_graph[n];
    d->saved_graph[n] = nullptr;
    d->saved_gexec[n] = nullptr;
    d->precision = n;
    // the persistent-kernel plan of this precision (host-side choices only)
    if (d->solver->ops && d->captured_gen == d->solver->ops_gen) CKR(d->setup_persistent());
    return SCFT_OK;
}

int scft_diblock_get_precision(scft_diblock_t d, int* out) {
    if (!d || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = d->precision;
    return SCFT_OK;
}

int scft_diblock_create(scft_solver_t s, double fA, double ds, double xN, double acceptance,
                        scft_diblock_t* out) {
    if (!s || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    if (!(fA > 0.0 && fA < 1.0)) return fail(SCFT_ERR_INVALID_ARG, "fA must be in (0,1)");
    if (!(ds > 0.0)) return fail(SCFT_ERR_INVALID_ARG, "ds must be > 0");
    // src/crysSCFT_sample.cpp:442-444 (truncating conversions)
    const double fB = 1 - fA;
    const size_t NsA = (size_t)(fA / ds);
    const size_t NsB = (size_t)(fB / ds);
    if (NsA < 1 || NsB < 1) return fail(SCFT_ERR_INVALID_ARG, "both blocks need at least one contour step");
    CK(cudaSetDevice(s->device));
    CKR(scft_solver_set_contour_step(s, ds));
    auto d = std::make_unique<scft_diblock_s>();
    d->solver = s;
    d->fA = fA; d->ds = ds; d->xN = xN; d->acc = acceptance;
    d->NsA = NsA; d->NsB = NsB; d->U = NsA + NsB; d->M = s->M;
    d->precision = s->precision;
    const size_t M = s->M;
    CKR(d->wA.alloc(M)); CKR(d->wB.alloc(M)); CKR(d->phiA.alloc(M)); CKR(d->phiB.alloc(M));
    CKR(d->ksi.alloc(M));
    CKR(d->partials.alloc(5 * kRedMaxBlocks));
    CKR(d->hist.alloc((size_t)d->hist_cap * HIST_STRIDE));
    CKR(d->state.alloc(1));
    CKR(zero_device(d->state.p, sizeof(IterState)));
    CKR(zero_device(d->phiA.p, M * sizeof(double)));
    CKR(zero_device(d->phiB.p, M * sizeof(double)));
    CKR(diblock_buffers(d.get(), d->precision));
    ++s->users;  // the solver outlives this context (scft_solver_destroy defers)
    *out = d.release();
    return SCFT_OK;
}

int scft_diblock_destroy(scft_diblock_t d) {
    if (!d) return SCFT_OK;
    scft_solver_t s = d->solver;
    cudaSetDevice(s->device);
    cudaStreamSynchronize(s->stream);
    delete d;
    --s->users;
    if (s->destroy_pending && s->users == 0) {
        s->destroy_pending = false;
        return scft_solver_destroy(s);
    }
    return SCFT_OK;
}

int scft_diblock_get_contour_counts(scft_diblock_t d, size_t* NsA, size_t* NsB) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (NsA) *NsA = d->NsA;
    if (NsB) *NsB = d->NsB;
    return SCFT_OK;
}

int scft_diblock_get_solver(scft_diblock_t d, scft_solver_t* out) {
    if (!d || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = d->solver;
    return SCFT_OK;
}

int scft_diblock_set_fields(scft_diblock_t d, const double* wA, const double* wB) {
    if (!d || !wA || !wB) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    CK(cudaSetDevice(d->solver->device));
    cudaStream_t st = d->solver->stream;
    CK(cudaMemcpyAsync(d->wA.p, wA, d->M * sizeof(double), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d->wB.p, wB, d->M * sizeof(double), cudaMemcpyHostToDevice, st));
    if (d->and_state.p) CK(cudaMemsetAsync(d->and_state.p, 0, sizeof(AndersonState), st));  // new fields: no history
    CK(cudaStreamSynchronize(st));
    d->fields_set = true;
    return SCFT_OK;
}

int scft_diblock_set_mixing(scft_diblock_t d, int history, double beta) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (history < 0 || history > kAndersonMax) return fail(SCFT_ERR_INVALID_ARG, "history must be in 0..32");
    if (history > 0 && !(beta > 0.0)) return fail(SCFT_ERR_INVALID_ARG, "beta must be > 0");
    CK(cudaSetDevice(d->solver->device));
    cudaStream_t st = d->solver->stream;
    CK(cudaStreamSynchronize(st));
    if (history > 0) {
        const size_t ring = (size_t)(history + 1) * 2 * d->M;
        if (d->and_W.n != ring) {
            CKR(d->and_W.alloc(ring));
            CKR(d->and_R.alloc(ring));
        }
        if (!d->and_partials.p) CKR(d->and_partials.alloc((size_t)kRedMaxBlocks * (kAndersonMax + 1)));
        if (!d->and_state.p) CKR(d->and_state.alloc(1));
        CK(cudaMemsetAsync(d->and_state.p, 0, sizeof(AndersonState), st));
        CK(cudaStreamSynchronize(st));
    }
    if (history != d->mix_history || beta != d->mix_beta) {
        // the captured iteration graphs (both precisions) embed the mixing kernels
        d->captured_gen = ~0ULL;
        d->saved_gen[0] = d->saved_gen[1] = ~0ULL;
    }
    d->mix_history = history;
    d->mix_beta = history > 0 ? beta : 0.0;
    return SCFT_OK;
}

int scft_diblock_set_wait_limit(scft_diblock_t d, long long spins) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (spins < 1) return fail(SCFT_ERR_INVALID_ARG, "the wait limit must be >= 1");
    CK(cudaSetDevice(d->solver->device));
    CK(cudaStreamSynchronize(d->solver->stream));
    if (spins != d->spin_limit) {
        // the limit is a kernel argument of the captured iteration graphs (both precisions)
        d->captured_gen = ~0ULL;
        d->saved_gen[0] = d->saved_gen[1] = ~0ULL;
        d->spin_limit = spins;
    }
    return SCFT_OK;
}

int scft_diblock_set_phi_form(scft_diblock_t d, int fused) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (fused != 0 && fused != 1) return fail(SCFT_ERR_INVALID_ARG, "phi form: 1 fused, 0 separate pass");
    CK(cudaSetDevice(d->solver->device));
    CK(cudaStreamSynchronize(d->solver->stream));
    if ((fused != 0) != d->fused_phi) {
        // the phi kernel is part of the captured FP64 iteration graph
        d->captured_gen = ~0ULL;
        d->saved_gen[0] = d->saved_gen[1] = ~0ULL;
        d->fused_phi = fused != 0;
    }
    return SCFT_OK;
}

int scft_diblock_get_residuals(scft_diblock_t d, double* out, size_t capacity, size_t* count) {
    if (!d || !count) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    const size_t n = d->last_residuals.size();
    *count = n;
    if (out) std::memcpy(out, d->last_residuals.data(), std::min(n, capacity) * sizeof(double));
    return SCFT_OK;
}

int scft_diblock_get_fields(scft_diblock_t d, double* phiA, double* phiB, double* wA, double* wB) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    CK(cudaSetDevice(d->solver->device));
    cudaStream_t st = d->solver->stream;
    const size_t b = d->M * sizeof(double);
    if (phiA) CK(cudaMemcpyAsync(phiA, d->phiA.p, b, cudaMemcpyDeviceToHost, st));
    if (phiB) CK(cudaMemcpyAsync(phiB, d->phiB.p, b, cudaMemcpyDeviceToHost, st));
    if (wA) CK(cudaMemcpyAsync(wA, d->wA.p, b, cudaMemcpyDeviceToHost, st));
    if (wB) CK(cudaMemcpyAsync(wB, d->wB.p, b, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return SCFT_OK;
}

int scft_diblock_stress(scft_diblock_t d, double dlnQ_dL[3], double* dF_dxN, double* Q_out) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (d->last_iter_precision != SCFT_FP64 && d->last_iter_precision != SCFT_FP32)
        return fail(SCFT_ERR_NOT_READY, "no iteration has run");
    // the contour of the last iteration: FP64, or FP32 after a precision-form iteration (its
    // values are promoted; the derivative triplets and the sums stay FP64)
    const bool f32 = d->last_iter_precision == SCFT_FP32;
    scft_solver_t s = d->solver;
    CK(cudaSetDevice(s->device));
    if (!s->ds_set || !s->ops || s->ds != d->ds) CKR(scft_solver_set_contour_step(s, d->ds));
    CKR(s->build_dops());
    cudaStream_t st = s->stream;
    const long long M = (long long)d->M;
    const long long U = (long long)d->U, NsA = (long long)d->NsA;
    IterState hs{};
    CK(cudaMemcpyAsync(&hs, d->state.p, sizeof(IterState), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    const double Q = hs.Q;
    if (!(Q > 0.0)) return fail(SCFT_ERR_NOT_READY, "no iteration has run");
    // slices per batch: about 64 MB per temporary field array
    long long tc = (64LL << 20) / (M * (long long)sizeof(double));
    if (tc < 1) tc = 1;
    if (tc > U) tc = U;
    if (d->stress_buf.n < (size_t)(4 * tc * M)) CKR(d->stress_buf.alloc((size_t)(4 * tc * M)));
    double* X = d->stress_buf.p;
    double* Y = X + tc * M;
    double* T1 = Y + tc * M;
    double* T2 = T1 + tc * M;
    const int rblocks = (int)std::min<long long>(kRedMaxBlocks, (tc * M + kRedThreads - 1) / kRedThreads);
    std::vector<double> part(kRedMaxBlocks);
    for (int ax = 0; ax < 3; ++ax) {
      double acc = 0.0;
      // d/dL_a of a sum of Kronecker products: the sum over terms of each term with its
      // axis-a factor replaced by the derivative factor
      for (int term = 0; term < s->ops->nterms; ++term) {
        const OpsSet* o = s->ops->term(term);
        const double* op[3];
        const double* opT[3];
        for (int b = 0; b < 3; ++b) {
            op[b] = b == ax ? o->d_dop[b].p : o->d_op[b].p;
            opT[b] = b == ax ? o->d_dopT[b].p : o->d_opT[b].p;
        }
        for (int blk = 0; blk < 2; ++blk) {
            const long long lo = blk == 0 ? 0 : NsA, hi = blk == 0 ? NsA : U;
            const double* D = blk == 0 ? d->d_wAds.p : d->d_wBds.p;
            const float* Df = blk == 0 ? d->f_wAds.p : d->f_wBds.p;
            for (long long t0 = lo; t0 < hi; t0 += tc) {
                const long long nt = std::min(tc, hi - t0);
                if (f32)
                    stress_scale_kernel<float><<<grid_blocks(nt * M, 256), 256, 0, st>>>(X, d->f_q.p, Df, t0, nt, M);
                else
                    stress_scale_kernel<double><<<grid_blocks(nt * M, 256), 256, 0, st>>>(X, d->d_q.p, D, t0, nt, M);
                CK(cudaGetLastError());
                CKR(s->triplet_batched(X, Y, T1, T2, nt, op, opT, st));
                const int nb = (int)std::min<long long>(rblocks, (nt * M + kRedThreads - 1) / kRedThreads);
                if (f32)
                    stress_dot_kernel<float><<<nb, kRedThreads, 0, st>>>(d->f_qc.p, Df, Y, t0, nt, M, d->partials.p);
                else
                    stress_dot_kernel<double><<<nb, kRedThreads, 0, st>>>(d->d_qc.p, D, Y, t0, nt, M, d->partials.p);
                CK(cudaGetLastError());
                CK(cudaMemcpyAsync(part.data(), d->partials.p, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                for (int i = 0; i < nb; ++i) acc += part[i];
            }
        }
      }
      if (dlnQ_dL) dlnQ_dL[ax] = acc / (double)M / Q;
    }
    if (dF_dxN) {
        // F (src/crysSCFT_sample.cpp:404-418) at fixed fields: d(xN <phiA phiB>)/dxN = <phiA phiB>,
        // and ksi = (wA + wB - xN)/2 gives d<-ksi (1 - phiA - phiB)>/dxN = <1 - phiA - phiB>/2
        const int nb = (int)std::min<long long>(kRedMaxBlocks, (M + kRedThreads - 1) / kRedThreads);
        dxn_terms_kernel<<<nb, kRedThreads, 0, st>>>(d->phiA.p, d->phiB.p, M, d->partials.p);
        CK(cudaGetLastError());
        std::vector<double> p2(2 * nb);
        CK(cudaMemcpyAsync(p2.data(), d->partials.p, p2.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        double ab = 0.0, inc = 0.0;
        for (int i = 0; i < nb; ++i) {
            ab += p2[2 * i];
            inc += p2[2 * i + 1];
        }
        *dF_dxN = ab / (double)M + 0.5 * inc / (double)M;
    }
    if (Q_out) *Q_out = Q;
    return SCFT_OK;
}

int scft_diblock_get_contour(scft_diblock_t d, int chain, size_t slot, double* out) {
    if (!d || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    if (chain != 0 && chain != 1) return fail(SCFT_ERR_INVALID_ARG, "chain must be 0 (q) or 1 (q+)");
    if (slot > d->U) return fail(SCFT_ERR_INVALID_ARG, "slot beyond NsA + NsB");
    CK(cudaSetDevice(d->solver->device));
    cudaStream_t st = d->solver->stream;
    const size_t M = d->M;
    if (d->precision == SCFT_FP64) {
        const double* src = (chain ? d->d_qc.p : d->d_q.p) + slot * M;
        CK(cudaMemcpyAsync(out, src, M * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    } else {
        std::vector<float> tmp(M);
        const float* src = (chain ? d->f_qc.p : d->f_q.p) + slot * M;
        CK(cudaMemcpyAsync(tmp.data(), src, M * sizeof(float), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        for (size_t i = 0; i < M; ++i) out[i] = tmp[i];
    }
    return SCFT_OK;
}

int scft_diblock_device_fields(scft_diblock_t d, double** phiA, double** phiB, double** wA, double** wB) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (phiA) *phiA = d->phiA.p;
    if (phiB) *phiB = d->phiB.p;
    if (wA) *wA = d->wA.p;
    if (wB) *wB = d->wB.p;
    d->fields_set = true;  // a caller that asks for device pointers may write the fields itself
    return SCFT_OK;
}

// Make the operators current and (re)build the launch plan when they changed.
static int diblock_prepare(scft_diblock_t d, bool want_graph) {
    if (!d->solver->ds_set || !d->solver->ops || d->solver->ds != d->ds)
        CKR(scft_solver_set_contour_step(d->solver, d->ds));
    if (d->captured_gen != d->solver->ops_gen) {
        if (d->gexec) cudaGraphExecDestroy(d->gexec);
        if (d->graph) cudaGraphDestroy(d->graph);
        d->gexec = nullptr;
        d->graph = nullptr;
        CKR(d->setup_persistent());
        d->captured_gen = d->solver->ops_gen;
    }
    if (want_graph) CKR(d->ensure_graph());
    return SCFT_OK;
}

// Clear and report device-side error bits e of the persistent kernel (0: none).
static int diblock_report_device_error(scft_diblock_t d, cudaStream_t st, unsigned e) {
    if (e) {
        CK(cudaMemsetAsync(d->ctrl.p + 1, 0, sizeof(unsigned), st));
        CK(cudaStreamSynchronize(st));
        if (e & 24u)
            return fail(SCFT_ERR_CUDA, "contour kernel: bulk-copy operand misaligned (error bits " + std::to_string(e) + ")");
        return fail(SCFT_ERR_TIMEOUT, "the contour kernel gave up waiting on a barrier, flag or bulk copy (error bits " +
                                          std::to_string(e) + ")");
    }
    return SCFT_OK;
}

// Read and clear the device-side error bits of the persistent kernel.
static int diblock_check_device_error(scft_diblock_t d, cudaStream_t st) {
    if (!d->ctrl.p) return SCFT_OK;
    unsigned e = 0;
    CK(cudaMemcpyAsync(&e, d->ctrl.p + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return diblock_report_device_error(d, st, e);
}

// Hand out `chunk` history rows h (iterations done .. done + chunk - 1) to the caller's
// arrays; false if an iteration flagged Q <= 0 or a non-finite free energy.
static bool diblock_take_history(scft_diblock_t d, const double* h, size_t chunk, size_t done, double* F,
                                 double* parts, double* maxinc, double* Q) {
    bool bad = false;
    for (size_t i = 0; i < chunk; ++i) {
        const double* r = &h[i * HIST_STRIDE];
        if (F) F[done + i] = r[HIST_F];
        if (parts) {
            parts[4 * (done + i) + 0] = r[HIST_EH];
            parts[4 * (done + i) + 1] = r[HIST_E0];
            parts[4 * (done + i) + 2] = r[HIST_E1];
            parts[4 * (done + i) + 3] = r[HIST_EK];
        }
        if (maxinc) maxinc[done + i] = r[HIST_MAXINC];
        if (Q) Q[done + i] = r[HIST_Q];
        d->last_residuals.push_back(r[HIST_RES]);
        if (r[HIST_FLAGS] != 0.0) bad = true;
    }
    return !bad;
}

static int diblock_run(scft_diblock_t d, size_t n_iter, double* F, double* parts, double* maxinc,
                       double* Q) {
    cudaStream_t st = d->solver->stream;
    CKR(diblock_prepare(d, true));
    size_t done = 0;
    std::vector<double> h;
    d->last_residuals.clear();
    while (done < n_iter) {
        const size_t chunk = std::min<size_t>(n_iter - done, d->hist_cap);
        IterState zero{};
        CK(cudaMemcpyAsync(d->state.p, &zero, sizeof(IterState), cudaMemcpyHostToDevice, st));
        for (size_t i = 0; i < chunk; ++i) CKR(d->run_once(st));
        h.resize(chunk * HIST_STRIDE);
        CK(cudaMemcpyAsync(h.data(), d->hist.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        CKR(diblock_check_device_error(d, st));
        if (chunk) d->last_iter_precision = d->precision;
        const bool ok = diblock_take_history(d, h.data(), chunk, done, F, parts, maxinc, Q);
        done += chunk;
        if (!ok) return fail(SCFT_ERR_NUMERIC, "Q <= 0 or a non-finite free energy in an iteration");
    }
    return SCFT_OK;
}

int scft_diblock_iterate(scft_diblock_t d, size_t n_iter, double* F, double* parts, double* maxinc,
                         double* Q) {
    if (!d) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    if (!d->fields_set) return fail(SCFT_ERR_NOT_READY, "set_fields first");
    CK(cudaSetDevice(d->solver->device));
    return diblock_run(d, n_iter, F, parts, maxinc, Q);
}

// Fields in, n_iter iterations, results out, all enqueued on the solver's stream with one
// synchronisation at the end (history rows and the error word through page-locked
// staging).  On an error the caller's phi/w arrays may already hold the failed
// iteration's values; the return code says so.
int scft_diblock_iterate_host(scft_diblock_t d, double* wA, double* wB, size_t n_iter, double* phiA,
                              double* phiB, double* F, double* parts, double* maxinc, double* Q) {
    if (!d || !wA || !wB) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    CK(cudaSetDevice(d->solver->device));
    if (n_iter > d->hist_cap) {  // more rows than one history buffer: the chunked path
        CKR(scft_diblock_set_fields(d, wA, wB));
        CKR(diblock_run(d, n_iter, F, parts, maxinc, Q));
        return scft_diblock_get_fields(d, phiA, phiB, wA, wB);
    }
    if (!d->pin_out) CK(cudaMallocHost(&d->pin_out, ((size_t)d->hist_cap * HIST_STRIDE + 1) * sizeof(double)));
    CKR(diblock_prepare(d, true));
    cudaStream_t st = d->solver->stream;
    const size_t b = d->M * sizeof(double);
    CK(cudaMemcpyAsync(d->wA.p, wA, b, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d->wB.p, wB, b, cudaMemcpyHostToDevice, st));
    if (d->and_state.p) CK(cudaMemsetAsync(d->and_state.p, 0, sizeof(AndersonState), st));  // new fields: no history
    d->fields_set = true;
    d->last_residuals.clear();
    CK(cudaMemsetAsync(d->state.p, 0, sizeof(IterState), st));
    for (size_t i = 0; i < n_iter; ++i) CKR(d->run_once(st));
    double* h = d->pin_out;
    unsigned* err = reinterpret_cast<unsigned*>(d->pin_out + (size_t)d->hist_cap * HIST_STRIDE);
    *err = 0;
    if (n_iter) CK(cudaMemcpyAsync(h, d->hist.p, n_iter * HIST_STRIDE * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (d->ctrl.p) CK(cudaMemcpyAsync(err, d->ctrl.p + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    if (phiA) CK(cudaMemcpyAsync(phiA, d->phiA.p, b, cudaMemcpyDeviceToHost, st));
    if (phiB) CK(cudaMemcpyAsync(phiB, d->phiB.p, b, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(wA, d->wA.p, b, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(wB, d->wB.p, b, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    CKR(diblock_report_device_error(d, st, *err));
    if (n_iter) d->last_iter_precision = d->precision;
    if (!diblock_take_history(d, h, n_iter, 0, F, parts, maxinc, Q))
        return fail(SCFT_ERR_NUMERIC, "Q <= 0 or a non-finite free energy in an iteration");
    return SCFT_OK;
}

int scft_diblock_launches_per_iteration(scft_diblock_t d, size_t* out) {
    if (!d || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = d->launches_per_iter;
    return SCFT_OK;
}

int scft_diblock_time_phases(scft_diblock_t d, size_t n_iter, double out[4]) {
    if (!d || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    if (!d->fields_set) return fail(SCFT_ERR_NOT_READY, "set_fields first");
    CK(cudaSetDevice(d->solver->device));
    CKR(diblock_prepare(d, false));
    cudaStream_t st = d->solver->stream;
    cudaEvent_t ev[5];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    double acc[4] = {0, 0, 0, 0};
    IterState zero{};
    CK(cudaMemcpyAsync(d->state.p, &zero, sizeof(IterState), cudaMemcpyHostToDevice, st));
    for (size_t it = 0; it < n_iter; ++it) {
        d->phase_events = ev;
        CK(cudaEventRecord(ev[0], st));
        CKR(d->enqueue(st));
        CK(cudaEventRecord(ev[4], st));
        CK(cudaEventSynchronize(ev[4]));
        float t01, t12, t23, t04;
        CK(cudaEventElapsedTime(&t01, ev[0], ev[1]));
        CK(cudaEventElapsedTime(&t12, ev[1], ev[2]));
        CK(cudaEventElapsedTime(&t23, ev[2], ev[3]));
        CK(cudaEventElapsedTime(&t04, ev[0], ev[4]));
        acc[0] += t04;
        acc[1] += t12;
        acc[2] += t23;
        acc[3] += t04 - t12 - t23;
        (void)t01;
    }
    d->phase_events = nullptr;
    for (auto& e : ev) cudaEventDestroy(e);
    for (int i = 0; i < 4; ++i) out[i] = n_iter ? acc[i] / (double)n_iter : 0.0;
    if (n_iter) d->last_iter_precision = d->precision;
    return diblock_check_device_error(d, st);
}

// ------------------------------- batches ----------------------------------
// Many independent SCFT instances (own grid, cell, fA, chiN): one solver and one
// iteration context each; one iteration of the whole batch is captured, fork-join over
// worker streams, into a single CUDA graph, so the instances' contour kernels run
// concurrently on the SMs.  The autotuner picks the number of worker streams and the
// contour-kernel form per batch by timing.
// ---------------------------------------------------------------------------
// Planner of the batch kernel (contour_batch.cuh): team sizes and CTA task lists.
// ---------------------------------------------------------------------------
// Cost model of one chain on a team of T CTAs (us), fitted to the batch kernel on a B200
// with every SM busy: per unit and phase 1.9 us of fixed work (tile fetch, waits, barriers,
// epilogue, stores) plus the axis products, ~1.02e-3 n^2 us; per phase one exchange
// (release, flag round trip) of ~2.3 us.
static double team_unit_us(int n) { return 1.9 + 1.02e-3 * (double)n * n; }
static double team_task_us(int n, int U, int T) { return (U + 1) * ((n / T) * team_unit_us(n) + 2.3); }

// First-fit decreasing of durations d into columns of capacity D: the column loads, or
// an empty vector if one duration exceeds D.  col[i] receives the column of item i.
static std::vector<double> pack_columns(const std::vector<double>& d, double D, std::vector<int>& col) {
    std::vector<size_t> order(d.size());
    for (size_t i = 0; i < d.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return d[x] > d[y]; });
    std::vector<double> load;
    col.assign(d.size(), -1);
    for (size_t i : order) {
        if (d[i] > D) return {};
        size_t c = 0;
        while (c < load.size() && load[c] + d[i] > D) ++c;
        if (c == load.size()) load.push_back(0.0);
        load[c] += d[i];
        col[i] = (int)c;
    }
    return load;
}

// Chains j (grid side n[j], U[j] steps) on G CTAs.  Chains of one grid side form a class;
// for a target makespan D a class with team size T runs in columns of T CTAs, its chains
// stacked in the columns by first-fit decreasing, and costs T x columns CTAs; every class
// takes the team size (a divisor of n, or the caller's fixed size) that costs fewest CTAs,
// and D is the smallest target (bisection) whose classes fit in G CTAs.  Every CTA belongs
// to one column and runs that column's chains in order, all CTAs of a column the same
// sequence, so no team ever waits for a CTA busy elsewhere.  Output: size[j]; tasks grouped
// by CTA (CTA b runs tasks[begin[b] .. begin[b+1]) in order); the planned makespan and the
// lower bound (team work / G), in us per iteration under the cost model.
static int team_schedule(const std::vector<int>& n, const std::vector<int>& U, int G,
                         const std::map<int, int>& fixed, std::vector<int>& size, std::vector<TeamTask>& tasks,
                         std::vector<int>& begin, double& planned, double& bound) {
    const size_t J = n.size();
    if (U.size() != J || G < 1) return fail(SCFT_ERR_INVALID_ARG, "team schedule: bad arguments");
    for (size_t j = 0; j < J; ++j)
        if (n[j] < 1 || U[j] < 1) return fail(SCFT_ERR_INVALID_ARG, "team schedule: bad chain");
    std::map<int, std::vector<size_t>> classes;
    for (size_t j = 0; j < J; ++j) classes[n[j]].push_back(j);
    std::map<int, std::vector<int>> cand;  // team sizes a class may take
    for (const auto& c : classes) {
        auto it = fixed.find(c.first);
        if (it != fixed.end()) {
            if (it->second < 1 || c.first % it->second || it->second > G)
                return fail(SCFT_ERR_INVALID_ARG, "team schedule: a fixed team size must divide the grid side and fit");
            cand[c.first] = {it->second};
        } else {
            for (int t = 1; t <= std::min(c.first, G); ++t)
                if (c.first % t == 0) cand[c.first].push_back(t);
        }
    }
    struct Choice {
        int T = 0;
        std::vector<double> load;
        std::vector<int> col;
    };
    // the cheapest choice of every class for target D; false if they need more than G CTAs
    auto plan_for = [&](double D, std::map<int, Choice>& out) {
        long long total = 0;
        for (const auto& c : classes) {
            Choice best;
            long long best_cost = -1;
            for (int T : cand[c.first]) {
                std::vector<double> d(c.second.size());
                for (size_t i = 0; i < d.size(); ++i) d[i] = team_task_us(c.first, U[c.second[i]], T);
                Choice ch;
                ch.T = T;
                ch.load = pack_columns(d, D, ch.col);
                if (ch.load.empty()) continue;
                const long long cost = (long long)T * ch.load.size();
                if (best_cost < 0 || cost < best_cost) {
                    best_cost = cost;
                    best = std::move(ch);
                }
            }
            if (best_cost < 0) return false;
            total += best_cost;
            out[c.first] = std::move(best);
        }
        return total <= G;
    };
    double hi = 0.0;
    for (size_t j = 0; j < J; ++j) hi += team_task_us(n[j], U[j], 1);
    std::map<int, Choice> plan;
    if (!plan_for(hi, plan)) {
        // more classes than CTAs: only then does one column per class not fit
        return fail(SCFT_ERR_UNSUPPORTED, "team schedule: more grid sizes than CTAs");
    }
    double lo = 0.0;
    for (int it = 0; it < 60; ++it) {
        const double mid = 0.5 * (lo + hi);
        std::map<int, Choice> p;
        if (plan_for(mid, p)) {
            hi = mid;
            plan = std::move(p);
        } else {
            lo = mid;
        }
    }
    // place the columns on consecutive CTAs; chains of a column run in FFD order
    size.assign(J, 1);
    struct Placed {
        double start;
        int chain, cta, rank, size;
    };
    std::vector<Placed> placed;
    int base = 0;
    planned = 0.0;
    bound = 0.0;
    for (const auto& c : classes) {
        const Choice& ch = plan[c.first];
        std::vector<double> t0(ch.load.size(), 0.0);
        std::vector<size_t> order(c.second.size());
        for (size_t i = 0; i < order.size(); ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
            return U[c.second[x]] > U[c.second[y]];  // FFD order: longest first within a column
        });
        for (size_t i : order) {
            const size_t j = c.second[i];
            const int col = ch.col[i];
            const double d = team_task_us(n[j], U[j], ch.T);
            size[j] = ch.T;
            for (int r = 0; r < ch.T; ++r) placed.push_back(Placed{t0[col], (int)j, base + col * ch.T + r, r, ch.T});
            t0[col] += d;
            bound += ch.T * d;
        }
        for (double l : t0) planned = std::max(planned, l);
        base += ch.T * (int)ch.load.size();
    }
    std::stable_sort(placed.begin(), placed.end(), [](const Placed& x, const Placed& y) {
        if (x.cta != y.cta) return x.cta < y.cta;
        if (x.start != y.start) return x.start < y.start;
        return x.chain < y.chain;
    });
    tasks.resize(placed.size());
    begin.assign(G + 1, 0);
    for (size_t t = 0; t < placed.size(); ++t) {
        tasks[t] = TeamTask{placed[t].chain, placed[t].rank, placed[t].size, 0};
        begin[placed[t].cta + 1]++;
    }
    for (int b = 0; b < G; ++b) begin[b + 1] += begin[b];
    bound /= G;
    return SCFT_OK;
}

struct scft_batch_s {
    int device = 0;
    std::vector<scft_solver_t> solvers;
    std::vector<scft_diblock_t> runs;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> joins;
    cudaStream_t main = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    size_t nstreams = 8;
    int form = 0;

    // Form 4: the contours of every instance whose own plan is the alternating FP64 kernel
    // run in ONE persistent launch of batch_contour_kernel (contour_batch.cuh); the
    // instances' prep and field kernels stay on the worker streams before and after it.
    std::map<int, int> team_fixed;  // grid side -> team size set by the caller (else the planner's choice)
    std::vector<char> in_team;      // per instance: its contour runs in the batch kernel
    DevBuf<TeamChain> team_chains;
    DevBuf<TeamTask> team_tasks;
    DevBuf<int> team_begin;
    DevBuf<unsigned> team_flags;    // every chain's exchange flags, zeroed before each launch
    DevBuf<unsigned> team_abort;
    int team_grid = 0;              // CTAs of the launch (0: no instance in the batch kernel)
    size_t team_smem = 0;
    size_t team_ntasks = 0;
    double team_planned_us = 0.0;   // makespan of the plan under the cost model
    double team_bound_us = 0.0;     // total team work / CTAs under the same model
    size_t launches = 0;            // kernel launches of one batch iteration

    // Team sizes, CTA assignment and device-side task lists of the batch kernel.
    int plan_teams() {
        const size_t n = runs.size();
        in_team.assign(n, 0);
        team_grid = 0;
        struct Ch {
            size_t run;
            int c, n, U, form;
        };
        std::vector<Ch> chs;
        size_t smem = 0;
        for (size_t i = 0; i < n; ++i) {
            scft_diblock_t d = runs[i];
            if (d->precision != SCFT_FP64 || !d->persistent || !d->alternating || !d->d_q.p || !d->ctrl.p) continue;
            const int side = (int)d->solver->grid_phy[0];
            const int f = team_form_for(side, d->solver->ops->eo[0] != 0, d->alt_eo2);
            if (f < 0) continue;
            in_team[i] = 1;
            smem = std::max(smem, team_form_smem(f));
            for (int c = 0; c < 2; ++c) chs.push_back(Ch{i, c, side, (int)d->U, f});
        }
        if (chs.empty()) return SCFT_OK;
        int sms = 0, dev_smem = 0;
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        CK(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        if (smem > (size_t)dev_smem) return fail(SCFT_ERR_UNSUPPORTED, "batch kernel: shared memory beyond the limit");
        CK(cudaFuncSetAttribute(batch_contour_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_contour_kernel, kContourThreads, smem));
        if (per_sm < 1) return fail(SCFT_ERR_UNSUPPORTED, "batch kernel: no block fits on a multiprocessor");
        const int G = per_sm * sms;

        std::vector<int> side(chs.size()), steps(chs.size()), size(chs.size());
        for (size_t j = 0; j < chs.size(); ++j) {
            side[j] = chs[j].n;
            steps[j] = chs[j].U;
        }
        std::vector<TeamTask> tasks;
        std::vector<int> begin;
        double planned = 0.0, bound = 0.0;
        CKR(team_schedule(side, steps, G, team_fixed, size, tasks, begin, planned, bound));

        // chain descriptors (tensor maps of each instance's stores and Boltzmann factors)
        size_t nflags = 0;
        std::vector<size_t> flag_off(chs.size());
        for (size_t j = 0; j < chs.size(); ++j) {
            flag_off[j] = nflags;
            nflags += 2 * (size_t)chs[j].n * chs[j].n;
        }
        CKR(team_flags.alloc(nflags));
        if (!team_abort.p) CKR(team_abort.alloc(1));
        std::vector<TeamChain> hc(chs.size());
        for (size_t j = 0; j < chs.size(); ++j) {
            const Ch& h = chs[j];
            scft_diblock_t d = runs[h.run];
            TeamChain& t = hc[j];
            std::memset(&t, 0, sizeof(TeamChain));
            double* q = h.c == 0 ? d->d_q.p : d->d_qc.p;
            for (int v = 0; v < 2; ++v) {  // plane [0] and slab [1] views, as launch_contour
                CKR(encode_panel_map(&t.tm_q[v], q, h.n, (long long)h.U + 1, v == 0));
                CKR(encode_panel_map(&t.tm_w[0][v], d->d_wAds.p, h.n, 0, v == 0));
                CKR(encode_panel_map(&t.tm_w[1][v], d->d_wBds.p, h.n, 0, v == 0));
            }
            t.q = q;
            t.xbuf = d->d_xch.p + (size_t)h.c * 2 * d->M;
            t.ops = d->alt_eo2 ? d->solver->ops->d_packed2.p : d->solver->ops->d_packed.p;
            t.flags = team_flags.p + flag_off[j];
            t.error = d->ctrl.p + 1;
            t.slot0 = h.c == 0 ? 0 : (long long)h.U;
            t.NsA = (long long)d->NsA;
            t.dir = h.c == 0 ? 1 : -1;
            t.U = h.U;
            t.n = h.n;
            t.form = h.form;
        }
        CKR(team_chains.alloc(hc.size()));
        CKR(team_tasks.alloc(tasks.size()));
        CKR(team_begin.alloc(begin.size()));
        CKR(upload(team_chains.p, hc.data(), hc.size() * sizeof(TeamChain)));
        CKR(upload(team_tasks.p, tasks.data(), tasks.size() * sizeof(TeamTask)));
        CKR(upload(team_begin.p, begin.data(), begin.size() * sizeof(int)));
        team_grid = G;
        team_smem = smem;
        team_ntasks = tasks.size();
        team_planned_us = planned;
        team_bound_us = bound;
        return SCFT_OK;
    }

    int launch_teams(cudaStream_t st) {
        CK(cudaMemsetAsync(team_flags.p, 0, team_flags.n * sizeof(unsigned), st));
        CK(cudaMemsetAsync(team_abort.p, 0, sizeof(unsigned), st));
        BatchContourArgs a{};
        a.chains = team_chains.p;
        a.tasks = team_tasks.p;
        a.task_begin = team_begin.p;
        a.abort = team_abort.p;
        a.spin_limit = runs[0]->spin_limit;  // the smallest wait limit of the instances
        for (auto d : runs) a.spin_limit = std::min(a.spin_limit, d->spin_limit);
        cudaLaunchConfig_t cfg{};
        cfg.gridDim = dim3((unsigned)team_grid);
        cfg.blockDim = dim3(kContourThreads);
        cfg.dynamicSmemBytes = team_smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CK(cudaLaunchKernelEx(&cfg, batch_contour_kernel, a));
        return SCFT_OK;
    }

    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
    }
    ~scft_batch_s() {
        if (main) cudaStreamSynchronize(main);
        drop_graph();
        for (auto r : runs) scft_diblock_destroy(r);
        for (auto s : solvers) scft_solver_destroy(s);
        for (auto e : joins) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        for (auto s : streams) cudaStreamDestroy(s);
        if (main) cudaStreamDestroy(main);
    }

    int make_streams(size_t ns) {
        for (auto e : joins) cudaEventDestroy(e);
        for (auto s : streams) cudaStreamDestroy(s);
        joins.clear();
        streams.clear();
        nstreams = std::max<size_t>(1, std::min(ns, runs.size()));
        for (size_t i = 0; i < nstreams; ++i) {
            cudaStream_t s;
            cudaEvent_t e;
            CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            streams.push_back(s);
            joins.push_back(e);
        }
        return SCFT_OK;
    }

    int build_graph() {
        drop_graph();
        const int ff = form == 4 ? 0 : form;  // the instances' own plan under form 4: automatic
        for (auto d : runs) {
            d->force_form = ff;
            if (d->captured_gen == d->solver->ops_gen && d->last_form != ff) d->captured_gen = ~0ULL;
            d->last_form = ff;
            CKR(diblock_prepare(d, false));
        }
        team_grid = 0;
        in_team.assign(runs.size(), 0);
        if (form == 4) CKR(plan_teams());
        const bool teams = team_grid > 0;
        using DB = scft_diblock_s;
        CK(cudaStreamBeginCapture(main, cudaStreamCaptureModeThreadLocal));
        int r = SCFT_OK;
        launches = 0;
        std::vector<size_t> pre(runs.size(), 0);
        cudaError_t e = cudaEventRecord(fork, main);
        for (size_t w = 0; w < nstreams && e == cudaSuccess; ++w) e = cudaStreamWaitEvent(streams[w], fork, 0);
        for (size_t i = 0; i < runs.size() && r == SCFT_OK && e == cudaSuccess; ++i) {
            r = runs[i]->enqueue(streams[i % nstreams], in_team[i] ? DB::kPartPrep : DB::kPartAll);
            pre[i] = runs[i]->launches_per_iter;
        }
        for (size_t w = 0; w < nstreams && e == cudaSuccess; ++w) {
            e = cudaEventRecord(joins[w], streams[w]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(main, joins[w], 0);
        }
        if (teams && r == SCFT_OK && e == cudaSuccess) {
            // one persistent launch: the contours of every instance in in_team
            r = launch_teams(main);
            ++launches;
            if (r == SCFT_OK) e = cudaEventRecord(fork, main);
            for (size_t w = 0; w < nstreams && e == cudaSuccess; ++w) e = cudaStreamWaitEvent(streams[w], fork, 0);
            for (size_t i = 0; i < runs.size() && r == SCFT_OK && e == cudaSuccess; ++i) {
                if (!in_team[i]) continue;
                r = runs[i]->enqueue(streams[i % nstreams], DB::kPartFields);
                runs[i]->launches_per_iter += pre[i];  // the instance's own kernels; the contour is counted once above
            }
            for (size_t w = 0; w < nstreams && e == cudaSuccess; ++w) {
                e = cudaEventRecord(joins[w], streams[w]);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(main, joins[w], 0);
            }
        }
        for (auto d : runs) launches += d->launches_per_iter;
        cudaGraph_t g = nullptr;
        const cudaError_t e2 = cudaStreamEndCapture(main, &g);
        if (r != SCFT_OK) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(SCFT_ERR_CUDA, std::string("batch capture: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
        }
        graph = g;
        CK(cudaGraphInstantiate(&gexec, graph, 0));
        return SCFT_OK;
    }

    // n_iter iterations; per-iteration F and max incompressibility of every instance
    int run(size_t n_iter, double* F, double* maxinc) {
        // rebuild when an instance's plan went stale (new operators, a new wait limit)
        bool stale = !gexec;
        for (auto d : runs) stale = stale || d->captured_gen != d->solver->ops_gen;
        if (stale) CKR(build_graph());
        const size_t n = runs.size();
        size_t done = 0;
        std::vector<double> h;
        while (done < n_iter) {
            const size_t chunk = std::min<size_t>(n_iter - done, 1024);
            IterState zero{};
            for (auto d : runs) CK(cudaMemcpyAsync(d->state.p, &zero, sizeof(IterState), cudaMemcpyHostToDevice, main));
            for (size_t k = 0; k < chunk; ++k) CK(cudaGraphLaunch(gexec, main));
            // device-side errors first (a kernel that gave up leaves unfinished fields, which
            // are not a numeric failure), every instance's word read and cleared
            {
                int first = SCFT_OK;
                std::string what;
                for (size_t i = 0; i < n; ++i) {
                    const int r = diblock_check_device_error(runs[i], main);
                    if (first == SCFT_OK && r != SCFT_OK) {
                        first = r;
                        what = "instance " + std::to_string(i) + " (grid " +
                               std::to_string(runs[i]->solver->grid_phy[0]) + ", batch form " + std::to_string(form) +
                               (i < in_team.size() && in_team[i] ? ", in the one launch" : ", own kernels") + "): " +
                               g_last_error;
                    }
                }
                if (first != SCFT_OK) return fail(first, what);
            }
            for (size_t i = 0; i < n; ++i) {
                scft_diblock_t d = runs[i];
                h.resize(chunk * HIST_STRIDE);
                CK(cudaMemcpyAsync(h.data(), d->hist.p, h.size() * sizeof(double), cudaMemcpyDeviceToHost, main));
                CK(cudaStreamSynchronize(main));
                for (size_t k = 0; k < chunk; ++k) {
                    const double* rr = &h[k * HIST_STRIDE];
                    if (F) F[(done + k) * n + i] = rr[HIST_F];
                    if (maxinc) maxinc[(done + k) * n + i] = rr[HIST_MAXINC];
                    if (rr[HIST_FLAGS] != 0.0) return fail(SCFT_ERR_NUMERIC, "instance " + std::to_string(i) + ": Q <= 0 or NaN");
                }
                d->last_iter_precision = d->precision;
            }
            done += chunk;
        }
        return SCFT_OK;
    }
};

int scft_batch_create(int kind, size_t n, const size_t* grid_log, const double* cell, const double* fA,
                      const double* xN, double ds, double acceptance, int precision, int device,
                      scft_batch_t* out) {
    if (!out || !grid_log || !cell || !fA || !xN || n == 0) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    auto b = std::make_unique<scft_batch_s>();
    if (device < 0) CK(cudaGetDevice(&device));
    b->device = device;
    for (size_t i = 0; i < n; ++i) {
        scft_solver_t s = nullptr;
        CKR(scft_solver_create(kind, grid_log + 3 * i, nullptr, precision, device, &s));
        b->solvers.push_back(s);
        const double c6[6] = {cell[3 * i], cell[3 * i + 1], cell[3 * i + 2], 0, 0, 0};
        CKR(scft_solver_set_cell_para(s, c6));
        scft_diblock_t d = nullptr;
        CKR(scft_diblock_create(s, fA[i], ds, xN[i], acceptance, &d));
        b->runs.push_back(d);
    }
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    CKR(b->make_streams(8));
    *out = b.release();
    return SCFT_OK;
}

int scft_batch_destroy(scft_batch_t b) {
    if (!b) return SCFT_OK;
    cudaSetDevice(b->device);
    delete b;
    return SCFT_OK;
}

int scft_batch_size(scft_batch_t b, size_t* n) {
    if (!b || !n) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    *n = b->runs.size();
    return SCFT_OK;
}

int scft_batch_instance(scft_batch_t b, size_t i, scft_diblock_t* d) {
    if (!b || !d || i >= b->runs.size()) return fail(SCFT_ERR_INVALID_ARG, "bad instance");
    *d = b->runs[i];
    return SCFT_OK;
}

int scft_batch_set_fields(scft_batch_t b, size_t i, const double* wA, const double* wB) {
    if (!b || i >= b->runs.size()) return fail(SCFT_ERR_INVALID_ARG, "bad instance");
    return scft_diblock_set_fields(b->runs[i], wA, wB);
}

int scft_batch_get_fields(scft_batch_t b, size_t i, double* phiA, double* phiB, double* wA, double* wB) {
    if (!b || i >= b->runs.size()) return fail(SCFT_ERR_INVALID_ARG, "bad instance");
    return scft_diblock_get_fields(b->runs[i], phiA, phiB, wA, wB);
}

int scft_batch_iterate(scft_batch_t b, size_t n_iter, double* F, double* maxinc) {
    if (!b) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    for (auto d : b->runs)
        if (!d->fields_set) return fail(SCFT_ERR_NOT_READY, "set the fields of every instance first");
    CK(cudaSetDevice(b->device));
    return b->run(n_iter, F, maxinc);
}

int scft_batch_configure(scft_batch_t b, size_t nstreams, int form) {
    if (!b || form < 0 || form > 4) return fail(SCFT_ERR_INVALID_ARG, "bad configuration");
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->main));
    b->drop_graph();
    b->form = form;
    return b->make_streams(nstreams);
}

int scft_batch_autotune(scft_batch_t b, size_t n_trial, size_t* best_nstreams, int* best_form, double* best_ms) {
    if (!b || n_trial == 0) return fail(SCFT_ERR_INVALID_ARG, "bad argument");
    CK(cudaSetDevice(b->device));
    const size_t n = b->runs.size();
    // The trials advance the fields and change the configuration.  A guard puts the
    // fields back and destroys the timing events on every exit; on an early (error) exit
    // it also restores the configuration the batch had before the call.
    struct Guard {
        scft_batch_t b;
        std::vector<std::vector<double>> keepA, keepB;
        size_t ns0;
        int form0;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        bool keep_config = false;
        ~Guard() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            cudaStreamSynchronize(b->main);
            if (!keep_config) scft_batch_configure(b, ns0, form0);
            for (size_t i = 0; i < keepA.size(); ++i)
                if (!keepA[i].empty()) scft_diblock_set_fields(b->runs[i], keepA[i].data(), keepB[i].data());
        }
    } g{b, std::vector<std::vector<double>>(n), std::vector<std::vector<double>>(n), b->nstreams, b->form};
    for (size_t i = 0; i < n; ++i) {
        std::vector<double> a(b->runs[i]->M), bb(b->runs[i]->M);
        CKR(scft_diblock_get_fields(b->runs[i], nullptr, nullptr, a.data(), bb.data()));
        g.keepA[i] = std::move(a);
        g.keepB[i] = std::move(bb);
    }
    CK(cudaEventCreate(&g.e0));
    CK(cudaEventCreate(&g.e1));
    double best = 1e300;
    size_t bs = b->nstreams;
    int bf = b->form;
    const size_t cand_streams[] = {2, 4, 8, 16, 32};
    const int cand_forms[] = {0, 2, 4};
    for (int f : cand_forms) {
        for (size_t ns : cand_streams) {
            if (ns > n && ns != cand_streams[0]) continue;
            // form 4: the worker streams only carry the small per-instance kernels
            if (f == 4 && ns != 4 && ns != 16) continue;
            CKR(scft_batch_configure(b, ns, f));
            CKR(b->run(1, nullptr, nullptr));  // capture + warm up
            CK(cudaEventRecord(g.e0, b->main));
            CKR(b->run(n_trial, nullptr, nullptr));
            CK(cudaEventRecord(g.e1, b->main));
            CK(cudaEventSynchronize(g.e1));
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, g.e0, g.e1));
            if (ms < best) {
                best = ms;
                bs = ns;
                bf = f;
            }
        }
    }
    CKR(scft_batch_configure(b, bs, bf));
    g.keep_config = true;  // the guard now only restores the fields and frees the events
    if (best_nstreams) *best_nstreams = bs;
    if (best_form) *best_form = bf;
    if (best_ms) *best_ms = best / (double)n_trial;
    return SCFT_OK;
}

int scft_team_schedule(size_t nchains, const int* n, const int* U, int G, size_t nfixed, const int* fixed_sides,
                       const int* fixed_sizes, int* size, size_t cap, int* task_chain, int* task_rank,
                       int* task_size, int* task_begin, size_t* ntasks, double* planned_us, double* bound_us) {
    if (!n || !U || !size || !task_begin || !ntasks || (nfixed && (!fixed_sides || !fixed_sizes)))
        return fail(SCFT_ERR_INVALID_ARG, "null argument");
    std::vector<int> vn(n, n + nchains), vu(U, U + nchains), sz;
    std::map<int, int> fixed;
    for (size_t i = 0; i < nfixed; ++i) fixed[fixed_sides[i]] = fixed_sizes[i];
    std::vector<TeamTask> tasks;
    std::vector<int> begin;
    double planned = 0.0, bound = 0.0;
    CKR(team_schedule(vn, vu, G, fixed, sz, tasks, begin, planned, bound));
    *ntasks = tasks.size();
    if (tasks.size() > cap || ((!task_chain || !task_rank || !task_size) && !tasks.empty()))
        return fail(SCFT_ERR_INVALID_ARG, "team schedule: task arrays too small (" + std::to_string(tasks.size()) +
                                              " tasks)");
    for (size_t j = 0; j < nchains; ++j) size[j] = sz[j];
    for (size_t t = 0; t < tasks.size(); ++t) {
        task_chain[t] = tasks[t].chain;
        task_rank[t] = tasks[t].rank;
        task_size[t] = tasks[t].size;
    }
    for (int b = 0; b <= G; ++b) task_begin[b] = begin[b];
    if (planned_us) *planned_us = planned;
    if (bound_us) *bound_us = bound;
    return SCFT_OK;
}

int scft_batch_set_team_sizes(scft_batch_t b, size_t count, const int* sides, const int* sizes) {
    if (!b || (count && (!sides || !sizes))) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    for (size_t i = 0; i < count; ++i)
        if (sides[i] < 1 || sizes[i] < 1 || sides[i] % sizes[i])
            return fail(SCFT_ERR_INVALID_ARG, "a team size must divide its grid side");
    CK(cudaSetDevice(b->device));
    CK(cudaStreamSynchronize(b->main));
    b->drop_graph();
    b->team_fixed.clear();
    for (size_t i = 0; i < count; ++i) b->team_fixed[sides[i]] = sizes[i];
    return SCFT_OK;
}

int scft_batch_team_plan(scft_batch_t b, int* grid, size_t* ntasks, size_t* ninstances, double* planned_us,
                         double* bound_us) {
    if (!b) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    CK(cudaSetDevice(b->device));
    if (!b->gexec) CKR(b->build_graph());
    size_t k = 0;
    for (char c : b->in_team) k += c ? 1 : 0;
    if (grid) *grid = b->team_grid;
    if (ntasks) *ntasks = b->team_grid ? b->team_ntasks : 0;
    if (ninstances) *ninstances = k;
    if (planned_us) *planned_us = b->team_grid ? b->team_planned_us : 0.0;
    if (bound_us) *bound_us = b->team_grid ? b->team_bound_us : 0.0;
    return SCFT_OK;
}

int scft_batch_launches_per_iteration(scft_batch_t b, size_t* out) {
    if (!b || !out) return fail(SCFT_ERR_INVALID_ARG, "null argument");
    CK(cudaSetDevice(b->device));
    if (!b->gexec) CKR(b->build_graph());
    *out = b->launches;
    return SCFT_OK;
}

int scft_solver_set_stream(scft_solver_t s, void* stream) {
    if (!s) return fail(SCFT_ERR_INVALID_ARG, "null handle");
    CK(cudaSetDevice(s->device));
    if (s->user_stream) CK(cudaStreamSynchronize(s->stream));
    if (!stream) {
        if (s->user_stream) s->stream = s->own_stream;
        s->user_stream = false;
    } else {
        CK(cudaStreamSynchronize(s->stream));
        s->stream = (cudaStream_t)stream;
        s->user_stream = true;
    }
    return SCFT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Triplet with library-owned static scratch (allocates nothing per call).
//
// For callers that cannot allocate device memory themselves or through us: an
// application whose device memory is entirely owned by another framework's pool
// (a fresh cudaMalloc could fail or fragment that pool), or a code path that must
// not run cudaMalloc/cudaFree because those calls can synchronise the device.
// The two intermediate fields of the three axis passes live in the file-scope
// array below instead of solver-owned cudaMalloc'd buffers.  Every GPU that loads
// this library holds the array (2 x SCFT_STATIC_SCRATCH_MAX_POINTS doubles, 4 MiB)
// until the process exits.
// ---------------------------------------------------------------------------
static __device__ __align__(256) double g_static_triplet_scratch[2 * SCFT_STATIC_SCRATCH_MAX_POINTS];

namespace {
constexpr int kMaxStaticDevices = 64;
std::mutex g_static_scratch_mu;
// device address of the array per ordinal, and the context it was looked up in: after a
// cudaDeviceReset the primary context (and with it the module holding the array) is
// created anew, so an address saved under the old context is looked up again
struct StaticScratchAddr {
    CUcontext ctx = nullptr;
    double* p = nullptr;
};
StaticScratchAddr g_static_scratch_dev[kMaxStaticDevices];

// cuCtxGetCurrent of the driver, resolved once (the library links the runtime only)
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
    });
    return fn;
}
}  // namespace

extern "C" int scft_solver_diffusion_device_static_scratch(scft_solver_t s, double* d_io, void* stream) {
    CKR(solver_ready(s));
    if (!d_io) return fail(SCFT_ERR_INVALID_ARG, "null buffer");
    if (s->M > (size_t)SCFT_STATIC_SCRATCH_MAX_POINTS)
        return fail(SCFT_ERR_INVALID_ARG,
                    "static-scratch triplet: space_size_phy " + std::to_string(s->M) + " exceeds the maximum " +
                        std::to_string((size_t)SCFT_STATIC_SCRATCH_MAX_POINTS));
    if (s->device < 0 || s->device >= kMaxStaticDevices)
        return fail(SCFT_ERR_INVALID_ARG, "static-scratch triplet: device ordinal out of range");
    // rejected before any device work, so a refused call never loads the module on its device
    if (s->ops->nterms > 1)
        return fail(SCFT_ERR_UNSUPPORTED,
                    "static-scratch triplet: a 3m solver with half-cell mirror translations needs a third scratch "
                    "field; use scft_solver_diffusion_device");
    CK(cudaSetDevice(s->device));
    double* scratch = nullptr;
    {
        // set-up once per device (and again after the device's context was replaced), with
        // that device current: the host-side name of the array is not a device address, so
        // ask the runtime for the address on this device
        CUcontext ctx = nullptr;
        CtxGetCurrentFn get_ctx = ctx_get_current();
        if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS)
            return fail(SCFT_ERR_CUDA, "static-scratch triplet: cuCtxGetCurrent is not available");
        std::lock_guard<std::mutex> lock(g_static_scratch_mu);
        StaticScratchAddr& a = g_static_scratch_dev[s->device];
        if (!a.p || a.ctx != ctx) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_static_triplet_scratch);
            if (e != cudaSuccess || !p)
                return fail(SCFT_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") +
                                               cudaGetErrorString(e));
            a.p = static_cast<double*>(p);
            a.ctx = ctx;
        }
        scratch = a.p;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : s->stream;
    // the z pass writes every element of t1 before the y pass reads it, and the y pass
    // writes every element of t2 before the x pass reads it: nothing needs clearing
    ChainIO<double> io[2] = {{d_io, d_io, nullptr, nullptr}, {}};
    double* t1[2] = {scratch, nullptr};
    double* t2[2] = {scratch + SCFT_STATIC_SCRATCH_MAX_POINTS, nullptr};
    return s->triplet<double>(1, io, t1, t2, st);
}
