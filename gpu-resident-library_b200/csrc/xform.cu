#include "xform.cuh"

#include "devonce.hpp"

namespace {

template <int LOGN, bool SINGLE>
cudaError_t launch_t(const xf::Job* jobs, const xf::Job* one, int njobs, bool inverse, cudaStream_t s) {
    using G = ntt::Geo<LOGN>;
    static gfx::DeviceOnce attrs;   // shared-memory limits, once per device
    attrs([] {
        cudaFuncSetAttribute(xf::k_fwd_col<LOGN, SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
        cudaFuncSetAttribute(xf::k_inv_col<LOGN, SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
        cudaFuncSetAttribute(xf::k_fwd_row<LOGN, SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
        cudaFuncSetAttribute(xf::k_inv_row<LOGN, SINGLE>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
    });
    const xf::Job o = one ? *one : xf::Job{};
    if (!inverse) {
        xf::k_fwd_col<LOGN, SINGLE><<<njobs * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(jobs, o);
        xf::k_fwd_row<LOGN, SINGLE><<<njobs * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(jobs, o);
    } else {
        xf::k_inv_row<LOGN, SINGLE><<<njobs * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(jobs, o);
        xf::k_inv_col<LOGN, SINGLE><<<njobs * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(jobs, o);
    }
    return cudaGetLastError();
}

template <int LOGN>
cudaError_t launch_lift(const xf::Job* jobs, int njobs, cudaStream_t s) {
    using G = ntt::Geo<LOGN>;
    static gfx::DeviceOnce attrs;
    attrs([] {
        cudaFuncSetAttribute(xf::k_fwd_col_lift<LOGN>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::COL_SMEM);
        cudaFuncSetAttribute(xf::k_fwd_row<LOGN, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::ROW_SMEM);
    });
    xf::k_fwd_col_lift<LOGN><<<njobs * G::COL_TILES, G::COL_THREADS, G::COL_SMEM, s>>>(jobs);
    xf::k_fwd_row<LOGN, false><<<njobs * G::ROW_TILES, G::ROW_THREADS, G::ROW_SMEM, s>>>(jobs, xf::Job{});
    return cudaGetLastError();
}

}  // namespace

bool xf_supported_logn(int logn) { return logn >= 9 && logn <= 16; }

cudaError_t xf_launch_ntt_lift(const xf::Job* jobs, int njobs, int logn, cudaStream_t s) {
    if (njobs <= 0) return cudaSuccess;
    switch (logn) {
        case 9: return launch_lift<9>(jobs, njobs, s);
        case 10: return launch_lift<10>(jobs, njobs, s);
        case 11: return launch_lift<11>(jobs, njobs, s);
        case 12: return launch_lift<12>(jobs, njobs, s);
        case 13: return launch_lift<13>(jobs, njobs, s);
        case 14: return launch_lift<14>(jobs, njobs, s);
        case 15: return launch_lift<15>(jobs, njobs, s);
        case 16: return launch_lift<16>(jobs, njobs, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t xf_launch_ntt(const xf::Job* jobs, const xf::Job* one, int njobs, int logn, bool inverse,
                          cudaStream_t s) {
    if (njobs <= 0) return cudaSuccess;
    switch (logn) {
        case 9: return one ? launch_t<9, true>(jobs, one, njobs, inverse, s) : launch_t<9, false>(jobs, one, njobs, inverse, s);
        case 10: return one ? launch_t<10, true>(jobs, one, njobs, inverse, s) : launch_t<10, false>(jobs, one, njobs, inverse, s);
        case 11: return one ? launch_t<11, true>(jobs, one, njobs, inverse, s) : launch_t<11, false>(jobs, one, njobs, inverse, s);
        case 12: return one ? launch_t<12, true>(jobs, one, njobs, inverse, s) : launch_t<12, false>(jobs, one, njobs, inverse, s);
        case 13: return one ? launch_t<13, true>(jobs, one, njobs, inverse, s) : launch_t<13, false>(jobs, one, njobs, inverse, s);
        case 14: return one ? launch_t<14, true>(jobs, one, njobs, inverse, s) : launch_t<14, false>(jobs, one, njobs, inverse, s);
        case 15: return one ? launch_t<15, true>(jobs, one, njobs, inverse, s) : launch_t<15, false>(jobs, one, njobs, inverse, s);
        case 16: return one ? launch_t<16, true>(jobs, one, njobs, inverse, s) : launch_t<16, false>(jobs, one, njobs, inverse, s);
        default: return cudaErrorInvalidValue;
    }
}
