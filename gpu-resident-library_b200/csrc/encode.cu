// Canonical CKKS encode / decode on the device (include/gpufhe_b200.h).
//
// The reference's encode_host / decode_host (src/encode.cpp:13-44) are O(N^2)
// host loops in double precision:
//   encode: m_j = llround((2 Delta / N) * sum_k (Re z_k Re tw[t] - Im z_k Im tw[t])),
//   decode: z_k = (sum_j m_j tw[t]) / Delta,     t = j * r_k mod 2N, r_k = 5^k mod 2N,
// with tw[t] = polar(1, -+pi t / N) from the host's libm. Here every output
// index is one thread that runs the same sum in the same order, with
// separately rounded products and sums (no fused multiply-add) and the
// twiddle table computed on the host by the same expression, so encodings and
// decodings equal the reference's bit for bit. A thread carries up to MB
// messages of a batch, so each twiddle gather (from the 2N-entry table in L2)
// serves MB sums.
#include <algorithm>
#include <cmath>
#include <complex>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "context.hpp"
#include "encode.h"
#include "gpufhe_b200.h"

struct gpufhe_encoder {
    uint32_t n = 0;
    int device = 0;
    double2* tw_enc = nullptr;   // [2n] polar(1, -pi t / n)
    double2* tw_dec = nullptr;   // [2n] polar(1, +pi t / n)
    uint32_t* r = nullptr;       // [n/2] 5^k mod 2n
    double2* ksi = nullptr;      // [2n] exp(2 pi i t / 2n), the fast transform's roots
};

namespace {

constexpr int ENT = 128;   // threads per block
constexpr int MB = 4;      // messages per thread

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// m[b][j], one thread per j, messages b0..b0+MB-1 of the batch.
__global__ void __launch_bounds__(ENT) k_encode(const double2* __restrict__ tw, const uint32_t* __restrict__ r,
                                                const double2* __restrict__ z, int64_t* __restrict__ m,
                                                uint32_t n, uint32_t count, double sc) {
    const uint32_t j = blockIdx.x * ENT + threadIdx.x;
    const uint32_t b0 = blockIdx.y * MB;
    if (j >= n) return;
    const uint32_t S = n / 2, mask = 2 * n - 1;
    const uint32_t nb = min((uint32_t)MB, count - b0);
    double acc[MB] = {0.0, 0.0, 0.0, 0.0};
    const double2* zb = z + (size_t)b0 * S;
#pragma unroll 4
    for (uint32_t k = 0; k < S; ++k) {
        const uint32_t t = (j * __ldg(r + k)) & mask;   // j * r_k mod 2n (2n divides 2^32)
        const double2 w = __ldg(tw + t);
#pragma unroll
        for (int b = 0; b < MB; ++b) {
            if (b < (int)nb) {
                const double2 v = __ldg(zb + (size_t)b * S + k);
                acc[b] = __dadd_rn(acc[b], __dsub_rn(__dmul_rn(v.x, w.x), __dmul_rn(v.y, w.y)));
            }
        }
    }
#pragma unroll
    for (int b = 0; b < MB; ++b)
        if (b < (int)nb) m[(size_t)(b0 + b) * n + j] = llround(__dmul_rn(sc, acc[b]));
}

// z[b][k], one thread per slot k.
__global__ void __launch_bounds__(ENT) k_decode(const double2* __restrict__ tw, const uint32_t* __restrict__ r,
                                                const int64_t* __restrict__ m, double2* __restrict__ z,
                                                uint32_t n, uint32_t count, double delta) {
    const uint32_t S = n / 2, mask = 2 * n - 1;
    const uint32_t k = blockIdx.x * ENT + threadIdx.x;
    const uint32_t b0 = blockIdx.y * MB;
    if (k >= S) return;
    const uint32_t nb = min((uint32_t)MB, count - b0);
    const uint32_t rk = __ldg(r + k);
    double ar[MB] = {0.0, 0.0, 0.0, 0.0}, ai[MB] = {0.0, 0.0, 0.0, 0.0};
    const int64_t* mb = m + (size_t)b0 * n;
#pragma unroll 4
    for (uint32_t j = 0; j < n; ++j) {
        const double2 w = __ldg(tw + ((j * rk) & mask));
#pragma unroll
        for (int b = 0; b < MB; ++b) {
            if (b < (int)nb) {
                const double mj = __ll2double_rn(__ldg(reinterpret_cast<const long long*>(mb) + (size_t)b * n + j));
                ar[b] = __dadd_rn(ar[b], __dmul_rn(mj, w.x));
                ai[b] = __dadd_rn(ai[b], __dmul_rn(mj, w.y));
            }
        }
    }
#pragma unroll
    for (int b = 0; b < MB; ++b)
        if (b < (int)nb) z[(size_t)(b0 + b) * S + k] = make_double2(__ddiv_rn(ar[b], delta), __ddiv_rn(ai[b], delta));
}

// ---------------------------------------------------------------- fast form
// The same maps by an O(n log n) transform over the rotation group (the
// "special" FFT of CKKS encoders): with S = n/2 and u_j = m_j + i m_{j+S},
//   decode: z_k = (sum_{j<S} u_j zeta^{j r_k}) / Delta, zeta = exp(i pi / n),
//   encode: u_j = (1/S) sum_k z_k zeta^{-j r_k}, m_j = Re u_j Delta,
//           m_{j+S} = Im u_j Delta,
// because zeta^{S r_k} = i for r_k = 1 mod 4. Radix-2 stages over the whole
// batch, one launch each (the batch stays in L2 between stages). Rounding
// differs from the reference's direct sums: coefficients may differ by one.
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

__global__ void k_bitrev(const double2* __restrict__ in, double2* __restrict__ out, uint32_t logS, size_t total) {
    const uint32_t S = 1u << logS;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t b = i >> logS;
        const uint32_t k = (uint32_t)(i & (S - 1));
        out[i] = in[(b << logS) + (__brev(k) >> (32 - logS))];
    }
}

// One stage of the forward (decode) transform, block length len:
// (u, v) -> (u + v ksi[(r_j mod 4 len) 2n / (4 len)], u - v ksi[...]).
__global__ void k_sfft_stage(double2* __restrict__ v, const uint32_t* __restrict__ r,
                             const double2* __restrict__ ksi, uint32_t logS, uint32_t len, uint32_t M,
                             size_t total) {
    const uint32_t lenh = len >> 1, lenq = len << 2;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t b = t >> (logS - 1);
        const uint32_t q = (uint32_t)(t & ((1u << (logS - 1)) - 1));
        const uint32_t j = q % lenh, i = (q / lenh) * len;
        double2* w = v + (b << logS) + i + j;
        const double2 a = w[0], c = cmul(w[lenh], __ldg(ksi + (size_t)(r[j] % lenq) * (M / lenq)));
        w[0] = make_double2(a.x + c.x, a.y + c.y);
        w[lenh] = make_double2(a.x - c.x, a.y - c.y);
    }
}

// One stage of the inverse (encode) transform:
// (u, v) -> (u + v, (u - v) ksi[(4 len - r_j mod 4 len) 2n / (4 len)]).
__global__ void k_sfft_inv_stage(double2* __restrict__ v, const uint32_t* __restrict__ r,
                                 const double2* __restrict__ ksi, uint32_t logS, uint32_t len, uint32_t M,
                                 size_t total) {
    const uint32_t lenh = len >> 1, lenq = len << 2;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t b = t >> (logS - 1);
        const uint32_t q = (uint32_t)(t & ((1u << (logS - 1)) - 1));
        const uint32_t j = q % lenh, i = (q / lenh) * len;
        double2* w = v + (b << logS) + i + j;
        const double2 a = w[0], c = w[lenh];
        w[0] = make_double2(a.x + c.x, a.y + c.y);
        w[lenh] = cmul(make_double2(a.x - c.x, a.y - c.y),
                       __ldg(ksi + (size_t)(lenq - r[j] % lenq) * (M / lenq)));
    }
}

// m_j = llround(Re u_j * sc), m_{j+S} = llround(Im u_j * sc), sc = Delta / S.
__global__ void k_fast_encode_out(const double2* __restrict__ u, int64_t* __restrict__ m, uint32_t logS, double sc,
                                  size_t total) {
    const uint32_t S = 1u << logS;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t b = i >> logS;
        const uint32_t j = (uint32_t)(i & (S - 1));
        const double2 x = u[i];
        m[(b << (logS + 1)) + j] = llround(x.x * sc);
        m[(b << (logS + 1)) + S + j] = llround(x.y * sc);
    }
}

// u_j = (m_j + i m_{j+S}) / Delta
__global__ void k_fast_decode_in(const int64_t* __restrict__ m, double2* __restrict__ u, uint32_t logS,
                                 double inv_delta, size_t total) {
    const uint32_t S = 1u << logS;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const size_t b = i >> logS;
        const uint32_t j = (uint32_t)(i & (S - 1));
        u[i] = make_double2((double)m[(b << (logS + 1)) + j] * inv_delta,
                            (double)m[(b << (logS + 1)) + S + j] * inv_delta);
    }
}

unsigned grid_of(size_t work) { return (unsigned)std::min<size_t>((work + 255) / 256, 148u * 32u); }

}  // namespace

extern "C" {

int gpufhe_encoder_create(uint32_t n, int device, gpufhe_encoder** out) {
    if (!out || n < 4 || (n & (n - 1)) || n > (1u << 17)) {
        gfx::set_error("gpufhe_encoder_create: n must be a power of two in [4, 2^17]");
        return GPUFHE_EINVAL;
    }
    *out = nullptr;
    int prev = 0;
    cudaGetDevice(&prev);
    auto* E = new gpufhe_encoder;
    try {
        ck(cudaSetDevice(device), "cudaSetDevice");
        E->n = n;
        E->device = device;
        const uint32_t M = 2 * n, S = n / 2;
        std::vector<double2> te(M), td(M);
        for (uint32_t t = 0; t < M; ++t) {
            // the reference's table expressions (encode.cpp:18, 35), host libm
            const std::complex<double> a = std::polar(1.0, -M_PI * (double)t / (double)n);
            const std::complex<double> b = std::polar(1.0, +M_PI * (double)t / (double)n);
            te[t] = make_double2(a.real(), a.imag());
            td[t] = make_double2(b.real(), b.imag());
        }
        std::vector<uint32_t> r(S);
        uint64_t rk = 1;
        for (uint32_t k = 0; k < S; ++k) { r[k] = (uint32_t)rk; rk = (rk * 5) % M; }
        std::vector<double2> ks(M);
        for (uint32_t t = 0; t < M; ++t) {
            const std::complex<double> w = std::polar(1.0, M_PI * (double)t / (double)n);
            ks[t] = make_double2(w.real(), w.imag());
        }
        ck(cudaMalloc(&E->ksi, M * sizeof(double2)), "cudaMalloc");
        ck(cudaMemcpy(E->ksi, ks.data(), M * sizeof(double2), cudaMemcpyHostToDevice), "upload");
        ck(cudaMalloc(&E->tw_enc, M * sizeof(double2)), "cudaMalloc");
        ck(cudaMalloc(&E->tw_dec, M * sizeof(double2)), "cudaMalloc");
        ck(cudaMalloc(&E->r, S * sizeof(uint32_t)), "cudaMalloc");
        ck(cudaMemcpy(E->tw_enc, te.data(), M * sizeof(double2), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemcpy(E->tw_dec, td.data(), M * sizeof(double2), cudaMemcpyHostToDevice), "upload");
        ck(cudaMemcpy(E->r, r.data(), S * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload");
    } catch (const std::exception& e) {
        gpufhe_encoder_destroy(E);
        cudaSetDevice(prev);
        gfx::set_error(e.what());
        return GPUFHE_ECUDA;
    }
    cudaSetDevice(prev);
    *out = E;
    return GPUFHE_OK;
}

void gpufhe_encoder_destroy(gpufhe_encoder* E) {
    if (!E) return;
    cudaFree(E->tw_enc);
    cudaFree(E->tw_dec);
    cudaFree(E->r);
    cudaFree(E->ksi);
    delete E;
}

int gpufhe_encode_batch_fast(gpufhe_encoder* E, uint32_t count, const double* z, double delta, int64_t* m,
                             cudaStream_t s) {
    if (!E || !z || !m) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    const uint32_t n = E->n, S = n / 2, M = 2 * n;
    uint32_t logS = 0;
    while ((1u << logS) < S) ++logS;
    if (logS < 1) { gfx::set_error("gpufhe_encode_batch_fast: n must be at least 4"); return GPUFHE_EINVAL; }
    const size_t words = (size_t)count * S;
    double2 *a = nullptr, *b = nullptr;
    int64_t* dm = nullptr;
    cudaError_t e = cudaMallocAsync(&a, words * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&b, words * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dm, (size_t)count * n * 8, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(a, z, words * sizeof(double2), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        for (uint32_t len = S; len >= 2; len >>= 1)
            k_sfft_inv_stage<<<grid_of(words / 2), 256, 0, s>>>(a, E->r, E->ksi, logS, len, M, words / 2);
        k_bitrev<<<grid_of(words), 256, 0, s>>>(a, b, logS, words);
        k_fast_encode_out<<<grid_of(words), 256, 0, s>>>(b, dm, logS, delta / (double)S, words);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(m, dm, (size_t)count * n * 8, cudaMemcpyDeviceToHost, s);
    for (void* p : {(void*)a, (void*)b, (void*)dm})
        if (p) cudaFreeAsync(p, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

int gpufhe_decode_batch_fast(gpufhe_encoder* E, uint32_t count, const int64_t* m, double delta, double* z,
                             cudaStream_t s) {
    if (!E || !z || !m) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    const uint32_t n = E->n, S = n / 2, M = 2 * n;
    uint32_t logS = 0;
    while ((1u << logS) < S) ++logS;
    if (logS < 1) { gfx::set_error("gpufhe_decode_batch_fast: n must be at least 4"); return GPUFHE_EINVAL; }
    const size_t words = (size_t)count * S;
    double2 *a = nullptr, *b = nullptr;
    int64_t* dm = nullptr;
    cudaError_t e = cudaMallocAsync(&a, words * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&b, words * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dm, (size_t)count * n * 8, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dm, m, (size_t)count * n * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        k_fast_decode_in<<<grid_of(words), 256, 0, s>>>(dm, a, logS, 1.0 / delta, words);
        k_bitrev<<<grid_of(words), 256, 0, s>>>(a, b, logS, words);
        for (uint32_t len = 2; len <= S; len <<= 1)
            k_sfft_stage<<<grid_of(words / 2), 256, 0, s>>>(b, E->r, E->ksi, logS, len, M, words / 2);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(z, b, words * sizeof(double2), cudaMemcpyDeviceToHost, s);
    for (void* p : {(void*)a, (void*)b, (void*)dm})
        if (p) cudaFreeAsync(p, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

int gpufhe_encode_batch(gpufhe_encoder* E, uint32_t count, const double* z, double delta, int64_t* m,
                        cudaStream_t s) {
    if (!E || !z || !m) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    const uint32_t n = E->n, S = n / 2;
    double2* dz = nullptr;
    int64_t* dm = nullptr;
    cudaError_t e = cudaMallocAsync(&dz, (size_t)count * S * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dm, (size_t)count * n * 8, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dz, z, (size_t)count * S * sizeof(double2), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        const double sc = 2.0 * delta / (double)n;   // encode.cpp:22
        k_encode<<<dim3((n + ENT - 1) / ENT, (count + MB - 1) / MB), ENT, 0, s>>>(E->tw_enc, E->r, dz, dm, n, count,
                                                                                 sc);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(m, dm, (size_t)count * n * 8, cudaMemcpyDeviceToHost, s);
    if (dz) cudaFreeAsync(dz, s);
    if (dm) cudaFreeAsync(dm, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

int gpufhe_decode_batch(gpufhe_encoder* E, uint32_t count, const int64_t* m, double delta, double* z,
                        cudaStream_t s) {
    if (!E || !z || !m) { gfx::set_error("null argument"); return GPUFHE_EINVAL; }
    if (!count) return GPUFHE_OK;
    const uint32_t n = E->n, S = n / 2;
    double2* dz = nullptr;
    int64_t* dm = nullptr;
    cudaError_t e = cudaMallocAsync(&dz, (size_t)count * S * sizeof(double2), s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dm, (size_t)count * n * 8, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dm, m, (size_t)count * n * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        k_decode<<<dim3((S + ENT - 1) / ENT, (count + MB - 1) / MB), ENT, 0, s>>>(E->tw_dec, E->r, dm, dz, n, count,
                                                                                 delta);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(z, dz, (size_t)count * S * sizeof(double2), cudaMemcpyDeviceToHost, s);
    if (dz) cudaFreeAsync(dz, s);
    if (dm) cudaFreeAsync(dm, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) { gfx::set_error(cudaGetErrorString(e)); return GPUFHE_ECUDA; }
    return GPUFHE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- reference C++ API
namespace {
// One encoder per (device, N) for the process; never freed (the reference's
// host functions hold no state, so callers expect none to manage).
gpufhe_encoder* encoder_for(uint32_t N) {
    static std::mutex mu;
    static std::map<std::pair<int, uint32_t>, gpufhe_encoder*> cache;
    int dev = 0;
    ck(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> g(mu);
    auto& e = cache[{dev, N}];
    if (!e && gpufhe_encoder_create(N, dev, &e) != GPUFHE_OK) {
        e = nullptr;
        throw std::runtime_error("encode_host: " + gfx::last_error());
    }
    return e;
}
}  // namespace

namespace gpufhe {

void encode_host(std::vector<int64_t>& m, const std::vector<std::complex<double>>& z, uint32_t N, double Delta) {
    if (z.size() < N / 2) throw std::invalid_argument("encode_host: z needs N/2 slots");
    m.assign(N, 0);
    // std::complex<double> is laid out as two doubles (re, im)
    if (gpufhe_encode_batch(encoder_for(N), 1, reinterpret_cast<const double*>(z.data()), Delta, m.data(), 0) !=
        GPUFHE_OK)
        throw std::runtime_error("encode_host: " + gfx::last_error());
}

void decode_host(std::vector<std::complex<double>>& z, const std::vector<int64_t>& m, uint32_t N, double Delta) {
    if (m.size() < N) throw std::invalid_argument("decode_host: m needs N coefficients");
    z.assign(N / 2, {0.0, 0.0});
    if (gpufhe_decode_batch(encoder_for(N), 1, m.data(), Delta, reinterpret_cast<double*>(z.data()), 0) !=
        GPUFHE_OK)
        throw std::runtime_error("decode_host: " + gfx::last_error());
}

}  // namespace gpufhe
