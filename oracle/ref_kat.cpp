/*
 * ref_kat.cpp -- TEST INFRASTRUCTURE ONLY: known-answer vectors from the
 * reference's OWN code.
 *
 * oracle/Makefile's `ref` target compiles this file with g++ against the
 * reference's headers exactly as they lie in the CrisOptix tree (never
 * copied into this repository): include/util/random.h,
 * include/graph/luminance.h, include/graph/restir/Reservoir.h,
 * include/graph/Camera.h, include/graph/CuBufferView.h,
 * include/model/Vertex.h and include/graph/sample_emitter.h whole, plus line
 * ranges cut unmodified by the recipe from files whose other parts need
 * OptiX: include/graph/restir/path_gen.h:12-72 (window constants, pairwise
 * MIS, SelectSpatialNeighbor, CalcReconnectionJacobian),
 * include/model/Emitter.h:6-55 (EmitterSample, EmitterData), and
 * shader/brdf.cu:12-37, 99-112 (PI, FresnelSchlick, D_GGX, V_SmithJointGGX).
 * oracle/ref_shim supplies a minimal glm and the CUDA qualifiers as nothing,
 * so the __host__ __device__ code runs on the host.  The output library,
 * oracle/_ref/libref_kat.so, pins the oracle: tests/golden/make_ref_kat.py
 * records its answers in tests/golden/ref_kat.npz, which the CPU suite checks
 * the oracle against and the GPU suite the CUDA device functions.
 */
#include <cstring>
#include <vector>

// the reference's headers, unmodified
#include <util/random.h>
#include <graph/luminance.h>
#include <graph/restir/Reservoir.h>
#include <graph/Camera.h>
#include <graph/CuBufferView.h>
#include <model/Vertex.h>

// unmodified line ranges of the reference, cut by the recipe into oracle/_ref/slices
#include "emitter_6_55.inc"
#include <graph/sample_emitter.h>
#include "path_gen_12_72.inc"
#include "brdf_12_37.inc"
#include "brdf_99_112.inc"

#include "kat.h"
#include "crisb.h"

namespace {

uint64_t get64(const uint32_t* w) { return static_cast<uint64_t>(w[0]) | (static_cast<uint64_t>(w[1]) << 32); }
void put64(uint32_t* w, uint64_t v) {
    w[0] = static_cast<uint32_t>(v);
    w[1] = static_cast<uint32_t>(v >> 32);
}
float getf(const uint32_t* w) {
    float f;
    std::memcpy(&f, w, 4);
    return f;
}
void putf(uint32_t* w, float f) { std::memcpy(w, &f, 4); }
glm::vec3 get3(const uint32_t* w) { return glm::vec3(getf(w), getf(w + 1), getf(w + 2)); }
void put3(uint32_t* w, const glm::vec3& v) {
    putf(w, v.x);
    putf(w + 1, v.y);
    putf(w + 2, v.z);
}
PCG32 rng_from(const uint32_t* w) {
    PCG32 r;
    r.state = get64(w);
    r.inc = get64(w + 2);
    return r;
}

struct KatSample {
    glm::vec3 f;
    uint32_t id = 0;
};

const int kIn[] = KAT_IN_WORDS;
const int kOut[] = KAT_OUT_WORDS;

void eval(int fn, const uint32_t* in, uint32_t* out) {
    switch (fn) {
        case KAT_TEA64:
            put64(out, SampleTEA64(in[0], in[1]));
            break;
        case KAT_PCG_SEED: {
            PCG32 r(get64(in), get64(in + 2));
            put64(out, r.state);
            put64(out + 2, r.inc);
            break;
        }
        case KAT_PCG_DRAWS: {
            PCG32 r = rng_from(in);
            out[0] = r.NextUint32();
            putf(out + 1, r.NextFloat());
            put64(out + 2, r.NextUint64());
            put64(out + 4, r.state);
            break;
        }
        case KAT_LUMINANCE:
            putf(out, GetLuminance(get3(in)));
            break;
        case KAT_MIS_CANON:
            putf(out, ComputeCanonicalPairwiseMISWeight(get3(in), get3(in + 3), getf(in + 6), getf(in + 7),
                                                        getf(in + 8), getf(in + 9)));
            break;
        case KAT_MIS_NEIGH:
            putf(out, ComputeNeighborPairwiseMISWeight(get3(in), get3(in + 3), getf(in + 6), getf(in + 7),
                                                       getf(in + 8), getf(in + 9)));
            break;
        case KAT_SELECT_NEIGHBOR: {
            PCG32 r = rng_from(in + 2);
            const glm::uvec2 n = SelectSpatialNeighbor(glm::uvec2(in[0], in[1]), r);
            out[0] = n.x;
            out[1] = n.y;
            put64(out + 2, r.state);
            break;
        }
        case KAT_JACOBIAN:
            putf(out, CalcReconnectionJacobian(get3(in), get3(in + 3), get3(in + 6), get3(in + 9)));
            break;
        case KAT_RESERVOIR: {
            PCG32 r = rng_from(in);
            Reservoir<KatSample> res;
            res.wSum = getf(in + 4);
            res.confidence = getf(in + 5);
            res.sample.f = get3(in + 6);
            res.sample.id = KAT_RES_STEPS;
            const uint32_t* c = in + 9;
            for (uint32_t s = 0; s < KAT_RES_STEPS; ++s, c += 5) {
                KatSample k;
                k.f = get3(c + 2);
                k.id = s;
                out[3 * s] = res.Update(k, getf(c), r, getf(c + 1)) ? 1u : 0u;
                putf(out + 3 * s + 1, res.wSum);
                putf(out + 3 * s + 2, res.confidence);
            }
            res.FinalizeGRIS();
            uint32_t* o = out + 3 * KAT_RES_STEPS;
            o[0] = res.sample.id;
            putf(o + 1, res.wSum);
            put64(o + 2, r.state);
            break;
        }
        case KAT_GGX: {
            putf(out, D_GGX(getf(in), getf(in + 3)));
            putf(out + 1, V_SmithJointGGX(getf(in + 1), getf(in + 2), getf(in + 3)));
            put3(out + 2, FresnelSchlick(get3(in + 5), getf(in + 4)));
            break;
        }
        case KAT_CAMERA_RAY: {
            CameraData cd;
            cd.pos = get3(in);
            cd.U = get3(in + 3);
            cd.V = get3(in + 6);
            cd.W = get3(in + 9);
            glm::vec3 o, d;
            SpawnCameraRay(cd, glm::vec2(getf(in + 12), getf(in + 13)), o, d);
            put3(out, d);
            break;
        }
        default:
            break;
    }
}

}  // namespace

extern "C" int ref_kat(int fn, const void* in, uint32_t n, void* out) {
    if (fn < 1 || fn > KAT_NUM_FN) return -1;
    const uint32_t* i = static_cast<const uint32_t*>(in);
    uint32_t* o = static_cast<uint32_t*>(out);
    for (uint32_t k = 0; k < n; ++k) eval(fn, i + static_cast<size_t>(k) * kIn[fn], o + static_cast<size_t>(k) * kOut[fn]);
    return 0;
}

/* SampleEmitter (sample_emitter.h:3-12) over a table built from crisb
 * emitters and world-space faces: n draws, draw k from PCG32 {states[2k],
 * states[2k + 1]}; out: 6 floats (point, colour), state_out: state after. */
extern "C" int ref_kat_emitter(const crisb_emitter* ems, uint32_t num_emitters, const float* faces, const uint64_t* states,
                               uint32_t n, float* out, uint64_t* state_out) {
    if (num_emitters == 0) return -1;
    std::vector<std::vector<Vertex>> verts(num_emitters);
    std::vector<std::vector<uint32_t>> idx(num_emitters);
    std::vector<EmitterData> table(num_emitters);
    for (uint32_t e = 0; e < num_emitters; ++e) {
        for (uint32_t f = 0; f < ems[e].num_faces; ++f)
            for (int c = 0; c < 3; ++c) {
                const float* p = faces + 9 * (static_cast<size_t>(ems[e].first_face) + f) + 3 * c;
                verts[e].push_back(Vertex(glm::vec3(p[0], p[1], p[2]), glm::vec3(0.0f), glm::vec3(0.0f), glm::vec2(0.0f)));
                idx[e].push_back(static_cast<uint32_t>(idx[e].size()));
            }
        EmitterData& d = table[e];
        d.color = glm::vec3(ems[e].color[0], ems[e].color[1], ems[e].color[2]);
        d.totalArea = 0.0f;
        d.vertexBuffer = CuBufferView<Vertex>(reinterpret_cast<CUdeviceptr>(verts[e].data()),
                                              static_cast<uint32_t>(verts[e].size()));
        d.indexBuffer = CuBufferView<uint32_t>(reinterpret_cast<CUdeviceptr>(idx[e].data()),
                                               static_cast<uint32_t>(idx[e].size()));
        d.areaCdfBuffer = CuBufferView<float>(0, ems[e].num_faces);  // only its count is read
    }
    const CuBufferView<EmitterData> view(reinterpret_cast<CUdeviceptr>(table.data()), num_emitters);
    for (uint32_t k = 0; k < n; ++k) {
        PCG32 r;
        r.state = states[2 * k];
        r.inc = states[2 * k + 1];
        const EmitterSample s = SampleEmitter(r, view);
        const float v[6] = {s.pos.x, s.pos.y, s.pos.z, s.color.x, s.color.y, s.color.z};
        std::memcpy(out + 6 * static_cast<size_t>(k), v, sizeof v);
        state_out[k] = r.state;
    }
    return 0;
}
