// records.cuh -- whole-record loads and stores of the device buffers and
// the image write shared by the pass kernels.
#pragma once

#include "pack16.cuh"
#include "passes.cuh"

namespace crisb {

RT_D uint32_t pixel_count(const FrameParams& fp) { return fp.width * fp.height; }

// Reservoir buffers in either storage layout (FP32 records or the packed
// FP16 records of pack16.cuh).  Whole-record access converts to the register
// form; the field readers touch only the words they need.
RT_D Res<Prefix> ld_pres(const PresBuf& b, uint32_t i) {
    if (b.f16) return unpack_pres16(ld_rec<crisb_prefix_res16_rec>(b.p, i));
    const crisb_prefix_res_rec r = ld_rec<crisb_prefix_res_rec>(b.p, i);
    return Res<Prefix>{ld_prefix(r.sample), r.w_sum, r.confidence};
}
RT_D void st_pres(const PresBuf& b, uint32_t i, const Res<Prefix>& r) {
    if (b.f16) {
        st_rec(b.p, i, pack_pres16(r));
        return;
    }
    crisb_prefix_res_rec o;
    st_prefix(o.sample, r.s);
    o.w_sum = r.w_sum;
    o.confidence = r.conf;
    o.pad[0] = 0;
    o.pad[1] = 0;
    st_rec(b.p, i, o);
}
RT_D uint32_t pres_flags(const PresBuf& b, uint32_t i) {
    return b.f16 ? static_cast<const crisb_prefix_res16_rec*>(b.p)[i].flags
                 : static_cast<const crisb_prefix_res_rec*>(b.p)[i].sample.flags;
}
RT_D float pres_wsum(const PresBuf& b, uint32_t i) {
    return b.f16 ? static_cast<const crisb_prefix_res16_rec*>(b.p)[i].w_sum
                 : static_cast<const crisb_prefix_res_rec*>(b.p)[i].w_sum;
}
RT_D float pres_conf(const PresBuf& b, uint32_t i) {
    return b.f16 ? static_cast<const crisb_prefix_res16_rec*>(b.p)[i].confidence
                 : static_cast<const crisb_prefix_res_rec*>(b.p)[i].confidence;
}
RT_D V3 pres_f(const PresBuf& b, uint32_t i) {
    return b.f16 ? unpack_rgb16(static_cast<const crisb_prefix_res16_rec*>(b.p)[i].f)
                 : ld3(static_cast<const crisb_prefix_res_rec*>(b.p)[i].sample.f);
}
RT_D Hit pres_last(const PresBuf& b, uint32_t i) {
    return b.f16 ? unpack_hit16(static_cast<const crisb_prefix_res16_rec*>(b.p)[i].last)
                 : ld_hit(static_cast<const crisb_prefix_res_rec*>(b.p)[i].sample.last);
}
RT_D Hit pres_primary(const PresBuf& b, uint32_t i) {
    return b.f16 ? unpack_hit16(static_cast<const crisb_prefix_res16_rec*>(b.p)[i].primary)
                 : ld_hit(static_cast<const crisb_prefix_res_rec*>(b.p)[i].sample.primary);
}
RT_D float pres_path_len(const PresBuf& b, uint32_t i) {
    return b.f16 ? static_cast<const crisb_prefix_res16_rec*>(b.p)[i].path_len
                 : static_cast<const crisb_prefix_res_rec*>(b.p)[i].sample.path_len;
}
// the record of pixel i of `src` into `dst` (same layout)
RT_D void copy_pres(const PresBuf& dst, const PresBuf& src, uint32_t i) {
    if (src.f16) st_rec(dst.p, i, ld_rec<crisb_prefix_res16_rec>(src.p, i));
    else st_rec(dst.p, i, ld_rec<crisb_prefix_res_rec>(src.p, i));
}

RT_D Res<Suffix> ld_sres(const SresBuf& b, uint32_t i) {
    if (b.f16) return unpack_sres16(ld_rec<crisb_suffix_res16_rec>(b.p, i));
    const crisb_suffix_res_rec r = ld_rec<crisb_suffix_res_rec>(b.p, i);
    return Res<Suffix>{ld_suffix(r.sample), r.w_sum, r.confidence};
}
RT_D void st_sres(const SresBuf& b, uint32_t i, const Res<Suffix>& r) {
    if (b.f16) {
        st_rec(b.p, i, pack_sres16(r));
        return;
    }
    crisb_suffix_res_rec o;
    st_suffix(o.sample, r.s);
    o.w_sum = r.w_sum;
    o.confidence = r.conf;
    st_rec(b.p, i, o);
}
RT_D uint32_t sres_flags(const SresBuf& b, uint32_t i) {
    return b.f16 ? static_cast<const crisb_suffix_res16_rec*>(b.p)[i].flags
                 : static_cast<const crisb_suffix_res_rec*>(b.p)[i].sample.flags;
}
RT_D Hit sres_last_prefix(const SresBuf& b, uint32_t i) {
    return b.f16 ? unpack_hit16(static_cast<const crisb_suffix_res16_rec*>(b.p)[i].last_prefix)
                 : ld_hit(static_cast<const crisb_suffix_res_rec*>(b.p)[i].sample.last_prefix);
}
RT_D V3 sres_f(const SresBuf& b, uint32_t i) {
    return b.f16 ? unpack_rgb16(static_cast<const crisb_suffix_res16_rec*>(b.p)[i].f)
                 : ld3(static_cast<const crisb_suffix_res_rec*>(b.p)[i].sample.f);
}
RT_D float sres_wsum(const SresBuf& b, uint32_t i) {
    return b.f16 ? static_cast<const crisb_suffix_res16_rec*>(b.p)[i].w_sum
                 : static_cast<const crisb_suffix_res_rec*>(b.p)[i].w_sum;
}
RT_D float sres_conf(const SresBuf& b, uint32_t i) {
    return b.f16 ? static_cast<const crisb_suffix_res16_rec*>(b.p)[i].confidence
                 : static_cast<const crisb_suffix_res_rec*>(b.p)[i].confidence;
}

// A suffix held either in an FP32 slot array (canonical records) or in a
// reservoir buffer.
struct SufRef {
    const crisb_suffix_res_rec* slot;  // non-null: FP32 slot array
    SresBuf res;
    uint32_t i;
};
RT_D Suffix ld_suf(const SufRef& r) { return r.slot ? ld_suffix(r.slot[r.i].sample) : ld_sres(r.res, r.i).s; }
RT_D Hit ld_suf_last(const SufRef& r) {
    return r.slot ? ld_hit(r.slot[r.i].sample.last_prefix) : sres_last_prefix(r.res, r.i);
}

// the FP32 slot records (canonical suffix, gather canonical suffix)
RT_D Res<Suffix> ld_sres(const crisb_suffix_res_rec* p, uint32_t i) {
    const crisb_suffix_res_rec r = ld_rec<crisb_suffix_res_rec>(p, i);
    return Res<Suffix>{ld_suffix(r.sample), r.w_sum, r.confidence};
}

RT_D void store_output(const FrameParams& fp, float* out, uint32_t i, V3 radiance) {
    V3 v = radiance;
    if (fp.p.enable_accum) {
        const V3 old = V3{out[3 * i], out[3 * i + 1], out[3 * i + 2]};
        const float blend = 1.0f / static_cast<float>(fp.frame_idx + 1);
        v = blend * radiance + (1.0f - blend) * old;
    }
    out[3 * i] = v.x;
    out[3 * i + 1] = v.y;
    out[3 * i + 2] = v.z;
}

// the per-pixel byte beside a suffix reservoir (kNval*): primary hit valid,
// prefix and canonical suffix valid for spatial reuse, sample valid
RT_D uint8_t nval_bits(bool primary_valid, bool spatial_ok, bool sample_valid) {
    if (!sample_valid) return 0;
    return static_cast<uint8_t>(kNvalSample | (primary_valid ? kNvalNeighbor : 0) | (spatial_ok ? kNvalSpatial : 0));
}

// ---- byte tally of the resampling kernels (statistics level 2) ----------------
// Each kernel adds the bytes of every field it reads or writes, at the size
// it is stored in, for the work actually present (valid neighbours, the
// chosen record); the sum over a frame is the roofline's algorithmic byte
// count.  A thread's count is added to its kernel's counter when the tally
// goes out of scope (one warp-aggregated atomic per exit point).
enum TallyKernel : int {
    kTallyPrefixCombine = 0,
    kTallyTemporalCombine = 1,
    kTallySpatialSelect = 2,
    kTallySpatialCombine = 3,
    kTallyGatherCombine = 4,
    kTallyKernels = 5
};

struct ByteTally {
    unsigned long long* counter;
    uint32_t n;
    RT_D ByteTally(const Bufs& b, int kernel) : counter(b.tally ? b.tally + kernel : nullptr), n(0) {}
    RT_D void add(uint32_t bytes) { n += bytes; }
    RT_D ~ByteTally() {
        if (!counter) return;
        const unsigned m = __activemask();
        const uint32_t sum = __reduce_add_sync(m, n);
        if ((threadIdx.x & 31) == __ffs(m) - 1) atomicAdd(counter, static_cast<unsigned long long>(sum));
    }
};

// stored sizes of reservoir records and of their weight fields (f, w_sum,
// confidence) in either storage layout
RT_D uint32_t pres_bytes(const PresBuf& b) {
    return b.f16 ? sizeof(crisb_prefix_res16_rec) : sizeof(crisb_prefix_res_rec);
}
RT_D uint32_t sres_bytes(const SresBuf& b) {
    return b.f16 ? sizeof(crisb_suffix_res16_rec) : sizeof(crisb_suffix_res_rec);
}
RT_D uint32_t weight_bytes(bool f16) { return (f16 ? 6u : 12u) + 8u; }

RT_D void invalidate(Res<Suffix>& r) {
    r.w_sum = 0.0f;
    r.conf = 0.0f;
    r.s.flags = fl_set_valid(r.s.flags, false);
}


}  // namespace crisb
