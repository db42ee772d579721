// selftest.cu -- crisb_selftest_kat: the library's device functions on packed
// known-answer records (oracle/kat.h layouts), one record per thread.  Tests
// compare the answers with those of the reference's own code; nothing on the
// rendering path calls this.
#include <string>

#include "radix_sort.h"
#include "rt_restir.cuh"

namespace crisb {

void set_last_error(const std::string& msg);

namespace {

// oracle/kat.h
constexpr int kKatNumFn = 11;
constexpr int kResSteps = 8;
__constant__ int kInWords[kKatNumFn + 1] = {0, 2, 4, 4, 3, 10, 10, 6, 12, 4 + 2 + 3 + 5 * kResSteps, 8, 14};
__constant__ int kOutWords[kKatNumFn + 1] = {0, 2, 4, 6, 1, 1, 1, 4, 1, 3 * kResSteps + 4, 5, 3};

RT_D uint64_t get64(const uint32_t* w) { return static_cast<uint64_t>(w[0]) | (static_cast<uint64_t>(w[1]) << 32); }
RT_D void put64(uint32_t* w, uint64_t v) {
    w[0] = static_cast<uint32_t>(v);
    w[1] = static_cast<uint32_t>(v >> 32);
}
RT_D float getf(const uint32_t* w) { return __uint_as_float(*w); }
RT_D void putf(uint32_t* w, float f) { *w = __float_as_uint(f); }
RT_D V3 get3(const uint32_t* w) { return V3{getf(w), getf(w + 1), getf(w + 2)}; }
RT_D void put3(uint32_t* w, V3 v) {
    putf(w, v.x);
    putf(w + 1, v.y);
    putf(w + 2, v.z);
}

struct KatSample {
    V3 f;
    uint32_t id;
};

// The library's PCG32 runs the default stream only (the reference never
// selects another): records with another increment are answered with all
// output words set to 0xFFFFFFFF and skipped by the tests.
__global__ void k_kat(int fn, const uint32_t* __restrict__ in_all, uint32_t n, uint32_t* __restrict__ out_all) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t* in = in_all + static_cast<size_t>(k) * kInWords[fn];
    uint32_t* out = out_all + static_cast<size_t>(k) * kOutWords[fn];
    auto default_stream = [](const uint32_t* w) { return get64(w + 2) == kPcgInc; };
    auto skip = [&]() {
        for (int i = 0; i < kOutWords[fn]; ++i) out[i] = 0xFFFFFFFFu;
    };
    switch (fn) {
        case 1:
            put64(out, tea64(in[0], in[1]));
            break;
        case 2: {
            if (get64(in + 2) != kPcgDefaultStream) return skip();
            const Rng r = rng_seeded(get64(in));
            put64(out, r.state);
            put64(out + 2, kPcgInc);
            break;
        }
        case 3: {
            if (!default_stream(in)) return skip();
            Rng r{get64(in)};
            out[0] = r.next_u32();
            putf(out + 1, r.next_float());
            put64(out + 2, r.next_u64());
            put64(out + 4, r.state);
            break;
        }
        case 4:
            putf(out, luminance(get3(in)));
            break;
        case 5:
            putf(out, mis_canonical(get3(in), get3(in + 3), getf(in + 6), getf(in + 7), getf(in + 8), getf(in + 9)));
            break;
        case 6:
            putf(out, mis_neighbor(get3(in), get3(in + 3), getf(in + 6), getf(in + 7), getf(in + 8), getf(in + 9)));
            break;
        case 7: {
            if (!default_stream(in + 2)) return skip();
            Rng r{get64(in + 2)};
            uint32_t nx = 0, ny = 0;
            select_spatial_neighbor(in[0], in[1], 10u, r, nx, ny);
            out[0] = nx;
            out[1] = ny;
            put64(out + 2, r.state);
            break;
        }
        case 8:
            putf(out, recon_jacobian(get3(in), get3(in + 3), get3(in + 6), get3(in + 9)));
            break;
        case 9: {
            if (!default_stream(in)) return skip();
            Rng r{get64(in)};
            Res<KatSample> res;
            res.w_sum = getf(in + 4);
            res.conf = getf(in + 5);
            res.s.f = get3(in + 6);
            res.s.id = kResSteps;
            const uint32_t* c = in + 9;
            for (int st = 0; st < kResSteps; ++st, c += 5) {
                const KatSample cand{get3(c + 2), static_cast<uint32_t>(st)};
                out[3 * st] = res_update(res, cand, getf(c), r, getf(c + 1)) ? 1u : 0u;
                putf(out + 3 * st + 1, res.w_sum);
                putf(out + 3 * st + 2, res.conf);
            }
            res_finalize(res);
            uint32_t* o = out + 3 * kResSteps;
            o[0] = res.s.id;
            putf(o + 1, res.w_sum);
            put64(o + 2, r.state);
            break;
        }
        case 10:
            putf(out, d_ggx(getf(in), getf(in + 3)));
            putf(out + 1, v_smith(getf(in + 1), getf(in + 2), getf(in + 3)));
            put3(out + 2, fresnel(get3(in + 5), getf(in + 4)));
            break;
        case 11:
            put3(out, spawn_camera_dir(get3(in + 3), get3(in + 6), get3(in + 9), getf(in + 12), getf(in + 13)));
            break;
        default:
            break;
    }
}

}  // namespace
}  // namespace crisb

extern "C" int crisb_selftest_kat(int fn, const void* in_dev, uint32_t n, void* out_dev, void* stream) {
    if (fn < 1 || fn > crisb::kKatNumFn || (n > 0 && (!in_dev || !out_dev))) {
        crisb::set_last_error("selftest: bad function id or null array");
        return CRISB_ERR_INVALID_ARGUMENT;
    }
    if (reinterpret_cast<uintptr_t>(in_dev) % 4 != 0 || reinterpret_cast<uintptr_t>(out_dev) % 4 != 0) {
        crisb::set_last_error("selftest: arrays must be 4-byte aligned");
        return CRISB_ERR_INVALID_ARGUMENT;
    }
    if (n == 0) return CRISB_OK;
    crisb::k_kat<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        fn, static_cast<const uint32_t*>(in_dev), n, static_cast<uint32_t*>(out_dev));
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        crisb::set_last_error(std::string("selftest: ") + cudaGetErrorString(e));
        return CRISB_ERR_CUDA;
    }
    return CRISB_OK;
}

extern "C" int crisb_selftest_sort(const uint64_t* in_dev, uint64_t* out_dev, uint32_t n, void* temp_dev,
                                   size_t temp_bytes, void* stream) {
    if (n > 0 && (!in_dev || !out_dev || !temp_dev || temp_bytes < crisb::rsort::temp_bytes(n))) {
        crisb::set_last_error("selftest sort: null array or scratch too small");
        return CRISB_ERR_INVALID_ARGUMENT;
    }
    const cudaError_t e =
        crisb::rsort::sort_high32(in_dev, out_dev, temp_dev, temp_bytes, n, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        crisb::set_last_error(std::string("selftest sort: ") + cudaGetErrorString(e));
        return CRISB_ERR_CUDA;
    }
    return CRISB_OK;
}

extern "C" size_t crisb_selftest_sort_temp_bytes(uint32_t n) { return crisb::rsort::temp_bytes(n); }
