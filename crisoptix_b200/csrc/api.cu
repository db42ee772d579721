// api.cu -- host side of the library: scene creation and device BVH build,
// the renderer and its frame orchestration, and the C ABI of include/crisb.h.
//
// Mirrors Scene (src/Scene.cpp), Camera::GetData (src/Camera.cpp:20-32) and
// Renderer (src/Renderer.cpp).  No call throws across the ABI; failures are
// status codes with a per-thread message (crisb_last_error).

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "bvh_device.h"
#include "passes.cuh"
#include "radix_sort.h"
#include "records.cuh"

namespace crisb {
namespace {

thread_local std::string g_last_error;

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        const int code = (e == cudaErrorMemoryAllocation) ? CRISB_ERR_OUT_OF_MEMORY : CRISB_ERR_CUDA;
        throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
void require(bool ok, const std::string& msg) {
    if (!ok) throw Error(CRISB_ERR_INVALID_ARGUMENT, msg);
}

template <typename F>
int guarded(F&& f) {
    try {
        f();
        return CRISB_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host allocation failed";
        return CRISB_ERR_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return CRISB_ERR_CUDA;
    }
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
    void alloc(size_t count) {
        release();
        if (count == 0) count = 1;
        check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
        n = count;
    }
    void upload(const T* src, size_t count) {
        alloc(count);
        if (count) check(cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice), "upload");
    }
    size_t bytes() const { return n * sizeof(T); }
};

// host PCG32 with an explicit stream (per-frame random of LaunchFrame)
uint32_t frame_random(uint64_t seed, uint64_t counter) {
    uint64_t state = 0;
    const uint64_t inc = (counter << 1u) | 1u;
    auto next = [&]() {
        const uint64_t old = state;
        state = old * kPcgMult + inc;
        const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
        const uint32_t rot = static_cast<uint32_t>(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    };
    next();
    state += seed;
    next();
    return next();
}

// Camera::GetData (src/Camera.cpp:20-32).  The rotation block of
// inverse(lookAt) is the transpose of lookAt's, so its columns (s, u, -f)
// are taken directly.
crisb_camera_data camera_data(const crisb_camera& c) {
    const V3 pos = ld3(c.pos), view = ld3(c.view_dir), up = ld3(c.up);
    const V3 center = pos + view;
    const V3 f = normalize(center - pos);
    const V3 s = normalize(cross(f, up));
    const V3 u = cross(s, f);
    const float tan_half = std::tan(0.5f * c.fov);
    crisb_camera_data d;
    st3(d.pos, pos);
    st3(d.u, normalize(s) * tan_half * c.aspect);
    st3(d.v, -normalize(u) * tan_half);
    st3(d.w, -normalize(-f));
    return d;
}

}  // namespace

// shared by the other translation units of the library
void set_last_error(const std::string& msg) { g_last_error = msg; }

__global__ void k_trace_rays(SceneView s, const float* rays, crisb_trace_hit* hits, uint32_t n, int any_hit) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* r = rays + 8 * static_cast<size_t>(i);
    const RayPre rp = make_ray(V3{r[0], r[1], r[2]}, V3{r[4], r[5], r[6]});
    crisb_trace_hit h;
    if (any_hit) {
        const TraceResult t = traverse<true>(s, rp, r[3], r[7]);
        h.prim = t.prim != CRISB_INVALID_PRIM ? 1u : 0u;
        h.t = h.u = h.v = 0.0f;
    } else {
        const TraceResult t = traverse<false>(s, rp, r[3], r[7]);
        h.prim = t.prim;
        h.t = t.prim != CRISB_INVALID_PRIM ? t.t : 0.0f;
        h.u = t.prim != CRISB_INVALID_PRIM ? t.u : 0.0f;
        h.v = t.prim != CRISB_INVALID_PRIM ? t.v : 0.0f;
    }
    hits[i] = h;
}

// default (never written) records: every hit invalid, everything else zero
__global__ void k_init_records(PresBuf pres0, PresBuf pres1, crisb_prefix_rec* cpre, SresBuf sres0, SresBuf sres1,
                               crisb_suffix_res_rec* csuf, crisb_gbuffer_rec* gbuf, uint32_t P) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P) return;
    crisb_prefix_res_rec pr;
    memset(&pr, 0, sizeof(pr));
    pr.sample.primary.prim = pr.sample.recon.prim = pr.sample.last.prim = CRISB_INVALID_PRIM;
    const Res<Prefix> rp{ld_prefix(pr.sample), 0.0f, 0.0f};
    st_pres(pres0, i, rp);
    st_pres(pres1, i, rp);
    cpre[i] = pr.sample;
    crisb_suffix_res_rec sr;
    memset(&sr, 0, sizeof(sr));
    sr.sample.recon.prim = sr.sample.last_prefix.prim = CRISB_INVALID_PRIM;
    const Res<Suffix> rs{ld_suffix(sr.sample), 0.0f, 0.0f};
    st_sres(sres0, i, rs);
    st_sres(sres1, i, rs);
    csuf[i] = sr;
    crisb_gbuffer_rec g;
    memset(&g, 0, sizeof(g));
    gbuf[i] = g;
}


struct LbvhStorage {
    DevBuf<uint64_t> keys_in, keys;
    DevBuf<int> inner_parent, leaf_parent, inner_left, inner_right, range_lo, range_hi, flags;
    DevBuf<lbvh::Box> inner_box, leaf_box;
    DevBuf<uint32_t> n, order;
    DevBuf<BvhNode> nodes;
    void alloc(uint32_t cap) {
        const size_t c = std::max<uint32_t>(cap, 2);
        keys_in.alloc(c);
        keys.alloc(c);
        inner_parent.alloc(c);
        leaf_parent.alloc(c);
        inner_left.alloc(c);
        inner_right.alloc(c);
        range_lo.alloc(c);
        range_hi.alloc(c);
        flags.alloc(c);
        inner_box.alloc(c);
        leaf_box.alloc(c);
        n.alloc(1);
        order.alloc(c);
        nodes.alloc(c);
    }
    lbvh::Work work(int* err) {
        lbvh::Work w;
        w.keys_in = keys_in.p;
        w.keys = keys.p;
        w.inner_parent = inner_parent.p;
        w.leaf_parent = leaf_parent.p;
        w.inner_left = inner_left.p;
        w.inner_right = inner_right.p;
        w.range_lo = range_lo.p;
        w.range_hi = range_hi.p;
        w.inner_box = inner_box.p;
        w.leaf_box = leaf_box.p;
        w.flags = flags.p;
        w.n = n.p;
        w.nodes = nodes.p;
        w.order = order.p;
        w.err = err;
        return w;
    }
};

}  // namespace crisb

using namespace crisb;

struct crisb_scene {
    int device = 0;
    uint32_t num_tris = 0;
    float scene_size = 0.0f;
    std::vector<float> h_pos, h_nrm;
    std::vector<uint32_t> h_mat;
    std::vector<float> h_uv;  // 6 per triangle when the scene has uvs
    DevBuf<Bvh4Node> nodes;
    DevBuf<Bvh8QNode> qnodes;  // the compressed tree, when built (then `nodes` is empty)
    int bvh_max_stack = 0, bvh_max_depth = 0;
    uint32_t bvh_inner_children = 0, bvh_leaf_children = 0;
    bool bvh_on_device = false;  // built by build_wide_bvh_device
    DevBuf<float4> tris;
    DevBuf<float4> shade;
    DevBuf<crisb_material> mats;
    DevBuf<crisb_emitter> emitters;
    DevBuf<float> emitter_faces;
    uint32_t num_emitters = 0;
    DevBuf<float2> uvs;
    DevBuf<int4> mat_tex;
    DevBuf<uint32_t> texels;
    DevBuf<uint4> tex_info;
    bool textured = false;
    DevBuf<int> err;

    SceneView view(int* err_word) const {
        SceneView v;
        v.nodes = nodes.p;
        v.qnodes = qnodes.p;
        v.tris = tris.p;
        v.shade = shade.p;
        v.mats = mats.p;
        v.emitters = emitters.p;
        v.emitter_faces = emitter_faces.p;
        v.num_emitters = num_emitters;
        v.num_tris = num_tris;
        v.err = err_word;
        v.ray_count = nullptr;
        v.trav_count = nullptr;
        if (textured) {
            v.uvs = uvs.p;
            v.mat_tex = mat_tex.p;
            v.texels = texels.p;
            v.tex_info = tex_info.p;
        }
        return v;
    }
};

namespace {

void flatten(const crisb_scene_desc& d, crisb_scene& s) {
    require(d.positions && d.indices && d.triangle_material && d.materials, "scene: null array");
    require(d.num_materials > 0, "scene: no materials");
    require(d.emitters && d.num_emitters > 0 && d.emitter_faces, "scene: at least one emitter is required");
    for (uint32_t t = 0; t < d.num_triangles; ++t) {
        for (int c = 0; c < 3; ++c) require(d.indices[3 * t + c] < d.num_vertices, "scene: index out of range");
        require(d.triangle_material[t] < d.num_materials, "scene: material index out of range");
    }
    for (uint32_t e = 0; e < d.num_emitters; ++e) {
        require(d.emitters[e].num_faces > 0, "scene: emitter without faces");
        require(static_cast<uint64_t>(d.emitters[e].first_face) + d.emitters[e].num_faces <= d.num_emitter_faces,
                "scene: emitter face range out of bounds");
    }
    auto corner = [&](uint32_t t, int c, const float* M, float* p, float* n) {
        const uint32_t vi = d.indices[3 * t + c];
        const float* v = d.positions + 3 * static_cast<size_t>(vi);
        float nn[3];
        if (d.normals) {
            const float* q = d.normals + 3 * static_cast<size_t>(vi);
            nn[0] = q[0];
            nn[1] = q[1];
            nn[2] = q[2];
        } else {
            const float* a = d.positions + 3 * static_cast<size_t>(d.indices[3 * t]);
            const float* b = d.positions + 3 * static_cast<size_t>(d.indices[3 * t + 1]);
            const float* cc = d.positions + 3 * static_cast<size_t>(d.indices[3 * t + 2]);
            const V3 fn = normalize(cross(V3{b[0] - a[0], b[1] - a[1], b[2] - a[2]},
                                          V3{cc[0] - a[0], cc[1] - a[1], cc[2] - a[2]}));
            nn[0] = fn.x;
            nn[1] = fn.y;
            nn[2] = fn.z;
        }
        if (!M) {
            std::memcpy(p, v, 12);
            std::memcpy(n, nn, 12);
            return;
        }
        double m[3][3];
        for (int r = 0; r < 3; ++r) {
            for (int cc2 = 0; cc2 < 3; ++cc2) m[r][cc2] = M[4 * r + cc2];
            p[r] = static_cast<float>(M[4 * r] * static_cast<double>(v[0]) + M[4 * r + 1] * static_cast<double>(v[1]) +
                                      M[4 * r + 2] * static_cast<double>(v[2]) + M[4 * r + 3]);
        }
        // normal transform: inverse transpose of the 3x3 block, renormalised
        const double det = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) -
                           m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                           m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
        require(det != 0.0, "scene: singular instance transform");
        double cof[3][3];
        cof[0][0] = m[1][1] * m[2][2] - m[1][2] * m[2][1];
        cof[0][1] = m[1][2] * m[2][0] - m[1][0] * m[2][2];
        cof[0][2] = m[1][0] * m[2][1] - m[1][1] * m[2][0];
        cof[1][0] = m[0][2] * m[2][1] - m[0][1] * m[2][2];
        cof[1][1] = m[0][0] * m[2][2] - m[0][2] * m[2][0];
        cof[1][2] = m[0][1] * m[2][0] - m[0][0] * m[2][1];
        cof[2][0] = m[0][1] * m[1][2] - m[0][2] * m[1][1];
        cof[2][1] = m[0][2] * m[1][0] - m[0][0] * m[1][2];
        cof[2][2] = m[0][0] * m[1][1] - m[0][1] * m[1][0];
        double o[3];
        for (int r = 0; r < 3; ++r) o[r] = (cof[r][0] * nn[0] + cof[r][1] * nn[1] + cof[r][2] * nn[2]) / det;
        const double len = std::sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
        for (int r = 0; r < 3; ++r) n[r] = static_cast<float>(len > 0 ? o[r] / len : o[r]);
    };
    auto emit = [&](uint32_t first, uint32_t count, const float* M, int32_t override_mat) {
        for (uint32_t t = first; t < first + count; ++t) {
            float p[9], n[9];
            for (int c = 0; c < 3; ++c) corner(t, c, M, p + 3 * c, n + 3 * c);
            s.h_pos.insert(s.h_pos.end(), p, p + 9);
            s.h_nrm.insert(s.h_nrm.end(), n, n + 9);
            s.h_mat.push_back(override_mat >= 0 ? static_cast<uint32_t>(override_mat) : d.triangle_material[t]);
            if (d.uvs)
                for (int c = 0; c < 3; ++c) {
                    const float* uv = d.uvs + 2 * static_cast<size_t>(d.indices[3 * t + c]);
                    s.h_uv.push_back(uv[0]);
                    s.h_uv.push_back(uv[1]);
                }
        }
    };
    if (d.num_instances == 0) {
        emit(0, d.num_triangles, nullptr, -1);
    } else {
        require(d.instances && d.meshes, "scene: instances need meshes");
        for (uint32_t i = 0; i < d.num_instances; ++i) {
            const crisb_instance& in = d.instances[i];
            require(in.mesh < d.num_meshes, "scene: instance mesh out of range");
            const crisb_mesh& m = d.meshes[in.mesh];
            require(static_cast<uint64_t>(m.first_triangle) + m.num_triangles <= d.num_triangles,
                    "scene: mesh triangle range out of bounds");
            require(in.material_override < static_cast<int32_t>(d.num_materials),
                    "scene: material override out of range");
            emit(m.first_triangle, m.num_triangles, in.transform, in.material_override);
        }
    }
    require(s.h_mat.size() < 0x7FFFFFFFu, "scene: too many triangles");
    s.num_tris = static_cast<uint32_t>(s.h_mat.size());
    // Scene::GetSceneSize (src/Scene.cpp:48-71): bounds start at the origin
    float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (size_t k = 0; k < s.h_pos.size(); k += 3)
        for (int a = 0; a < 3; ++a) {
            lo[a] = gmin(lo[a], s.h_pos[k + a]);
            hi[a] = gmax(hi[a], s.h_pos[k + a]);
        }
    s.scene_size = distance(V3{lo[0], lo[1], lo[2]}, V3{hi[0], hi[1], hi[2]});
}

// Textures, their per-material assignment and the corner uvs (only when a
// material uses a texture).  Texels are packed RGBA8 words, one texture after
// the other.
void upload_textures(const crisb_scene_desc& d, crisb_scene& s) {
    if (!d.material_textures) return;
    std::vector<int4> mt(d.num_materials);
    bool any = false;
    for (uint32_t m = 0; m < d.num_materials; ++m) {
        int t[3];
        for (int k = 0; k < 3; ++k) {
            t[k] = d.material_textures[3 * m + k];
            require(t[k] >= -1 && t[k] < static_cast<int64_t>(d.num_textures), "scene: texture index out of range");
            any = any || t[k] >= 0;
        }
        mt[m] = make_int4(t[0], t[1], t[2], -1);
    }
    if (!any) return;
    require(d.uvs != nullptr, "scene: textured materials need uvs");
    require(d.textures != nullptr, "scene: null texture array");
    std::vector<uint4> info(d.num_textures);
    size_t words = 0;
    for (uint32_t t = 0; t < d.num_textures; ++t) {
        const crisb_texture& tx = d.textures[t];
        require(tx.rgba && tx.width > 0 && tx.height > 0 && tx.width < 65536 && tx.height < 65536,
                "scene: bad texture");
        require(words + static_cast<size_t>(tx.width) * tx.height < 0xffffffffu, "scene: textures too large");
        info[t] = make_uint4(static_cast<uint32_t>(words), tx.width, tx.height, 0);
        words += static_cast<size_t>(tx.width) * tx.height;
    }
    std::vector<uint32_t> texels(std::max<size_t>(words, 1));
    for (uint32_t t = 0; t < d.num_textures; ++t)
        std::memcpy(texels.data() + info[t].x, d.textures[t].rgba,
                    4 * static_cast<size_t>(d.textures[t].width) * d.textures[t].height);
    std::vector<float2> uv(3 * static_cast<size_t>(std::max<uint32_t>(s.num_tris, 1)), make_float2(0, 0));
    for (size_t k = 0; k < 3 * static_cast<size_t>(s.num_tris); ++k) uv[k] = make_float2(s.h_uv[2 * k], s.h_uv[2 * k + 1]);
    s.uvs.upload(uv.data(), uv.size());
    s.mat_tex.upload(mt.data(), mt.size());
    s.texels.upload(texels.data(), texels.size());
    s.tex_info.upload(info.data(), info.size());
    s.textured = true;
}

// The scene BVH built on the device (bvh_device.h), then copied back once for
// the same structural check as a host-built tree (every triangle in one leaf,
// boxes containing their subtrees, the traversal stack bound).  Returns false
// when the tree would need a deeper traversal stack than the kernels have
// (the host builder's median fallback then bounds the depth).
// child slots holding a node / triangles
void count_children(const std::vector<Bvh8QNode>& nodes, crisb_scene& s) {
    s.bvh_inner_children = s.bvh_leaf_children = 0;
    for (const Bvh8QNode& nd : nodes)
        for (int c = 0; c < 8; ++c) {
            if (nd.meta[c] == 0) continue;
            if ((nd.meta[c] & 0x18u) == 0x18u) ++s.bvh_inner_children;
            else ++s.bvh_leaf_children;
        }
}
void count_children(const std::vector<Bvh4Node>& nodes, crisb_scene& s) {
    s.bvh_inner_children = s.bvh_leaf_children = 0;
    for (const Bvh4Node& nd : nodes)
        for (int c = 0; c < kBvhWidth; ++c) {
            if (nd.link[c] == kNoChild) continue;
            if (nd.link[c] >= 0) ++s.bvh_inner_children;
            else ++s.bvh_leaf_children;
        }
}

// the compressed 8-wide tree on the device, validated on the host; false
// when the scene does not qualify (coordinates too large, tree deeper than
// the group stack)
bool build_qbvh_on_device(crisb_scene& s, float max_abs) {
    if (!(max_abs < kQMaxCoord)) return false;
    const uint32_t n = s.num_tris;
    DevBuf<float> pos;
    pos.upload(s.h_pos.data(), std::max<size_t>(s.h_pos.size(), 1));
    DeviceWideBvh db;
    const float margin = box_margin(max_abs);
    check(build_wide_bvh_device(pos.p, n, kQLeafMax, margin, true, nullptr, &db), "device BVH build");
    std::vector<Bvh8QNode> hn(db.num_nodes);
    std::vector<float4> t3(3 * static_cast<size_t>(std::max<uint32_t>(n, 1)));
    cudaError_t e = cudaMemcpy(hn.data(), db.qnodes, db.num_nodes * sizeof(Bvh8QNode), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(t3.data(), db.tris, t3.size() * sizeof(float4), cudaMemcpyDeviceToHost);
    auto drop = [&]() {
        cudaFree(db.qnodes);
        cudaFree(db.tris);
    };
    if (e != cudaSuccess) {
        drop();
        check(e, "device BVH copy");
    }
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) std::memcpy(&order[i], &t3[3 * i + 2].w, 4);
    int depth = 0;
    try {
        depth = validate_qbvh(hn, order, s.h_pos.data(), n, margin);
    } catch (const std::runtime_error& ex) {
        drop();
        throw Error(CRISB_ERR_INVALID_ARGUMENT, std::string("device scene build: ") + ex.what());
    }
    // at most one waiting group per level above the deepest node
    if (depth > kQStack) {
        drop();
        return false;
    }
    s.nodes.release();
    s.qnodes.release();
    s.qnodes.p = db.qnodes;
    s.qnodes.n = db.num_nodes;
    s.tris.release();
    s.tris.p = db.tris;
    s.tris.n = 3 * static_cast<size_t>(std::max<uint32_t>(n, 1));
    s.bvh_max_stack = depth;
    count_children(hn, s);
    s.bvh_max_depth = db.binary_depth;
    s.bvh_on_device = true;
    check(cudaDeviceSynchronize(), "scene build");
    return true;
}

bool build_bvh_on_device(crisb_scene& s) {
    const uint32_t n = s.num_tris;
    float max_abs = 0.0f;
    for (float v : s.h_pos) max_abs = std::max(max_abs, std::fabs(v));
    DevBuf<float> pos;
    pos.upload(s.h_pos.data(), std::max<size_t>(s.h_pos.size(), 1));
    DeviceWideBvh db;
    check(build_wide_bvh_device(pos.p, n, kTriLeafMax, box_margin(max_abs), false, nullptr, &db),
          "device BVH build");
    WideBvh hb;
    hb.nodes.resize(db.num_nodes);
    std::vector<float4> t3(3 * static_cast<size_t>(std::max<uint32_t>(n, 1)));
    cudaError_t e = cudaMemcpy(hb.nodes.data(), db.nodes, db.num_nodes * sizeof(Bvh4Node), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(t3.data(), db.tris, t3.size() * sizeof(float4), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaFree(db.nodes);
        cudaFree(db.tris);
        check(e, "device BVH copy");
    }
    hb.order.resize(n);
    for (uint32_t i = 0; i < n; ++i) std::memcpy(&hb.order[i], &t3[3 * i + 2].w, 4);
    hb.max_stack = 1 << 30;
    int stack = 0;
    try {
        stack = validate_wide_bvh(hb, s.h_pos.data(), n, kTriLeafMax);
    } catch (const std::runtime_error& ex) {
        cudaFree(db.nodes);
        cudaFree(db.tris);
        throw Error(CRISB_ERR_INVALID_ARGUMENT, std::string("device scene build: ") + ex.what());
    }
    if (stack > kTraversalStack) {
        cudaFree(db.nodes);
        cudaFree(db.tris);
        return false;
    }
    s.nodes.release();
    s.nodes.p = db.nodes;
    s.nodes.n = db.num_nodes;
    s.tris.release();
    s.tris.p = db.tris;
    s.tris.n = 3 * static_cast<size_t>(std::max<uint32_t>(n, 1));
    s.bvh_max_stack = stack;
    count_children(hb.nodes, s);
    s.bvh_max_depth = db.binary_depth;
    s.bvh_on_device = true;
    check(cudaDeviceSynchronize(), "scene build");
    return true;
}

void build_scene(const crisb_scene_desc& d, crisb_scene& s) {
    check(cudaGetDevice(&s.device), "cudaGetDevice");
    flatten(d, s);
    const uint32_t n = s.num_tris;
    // shading records: p0 p1 p2 n0 n1 n2 material (5 float4 per triangle)
    std::vector<float4> shade(5 * static_cast<size_t>(std::max<uint32_t>(n, 1)));
    for (uint32_t t = 0; t < n; ++t) {
        const float* p = &s.h_pos[9 * static_cast<size_t>(t)];
        const float* q = &s.h_nrm[9 * static_cast<size_t>(t)];
        float m;
        std::memcpy(&m, &s.h_mat[t], 4);
        shade[5 * t + 0] = make_float4(p[0], p[1], p[2], p[3]);
        shade[5 * t + 1] = make_float4(p[4], p[5], p[6], p[7]);
        shade[5 * t + 2] = make_float4(p[8], q[0], q[1], q[2]);
        shade[5 * t + 3] = make_float4(q[3], q[4], q[5], q[6]);
        shade[5 * t + 4] = make_float4(q[7], q[8], m, 0.0f);
    }
    s.shade.upload(shade.data(), shade.size());
    s.mats.upload(d.materials, d.num_materials);
    s.emitters.upload(d.emitters, d.num_emitters);
    s.emitter_faces.upload(d.emitter_faces, 9 * static_cast<size_t>(d.num_emitter_faces));
    s.num_emitters = d.num_emitters;
    upload_textures(d, s);
    s.err.alloc(1);
    check(cudaMemset(s.err.p, 0, sizeof(int)), "memset");
    require(d.bvh_builder == CRISB_BVH_DEVICE || d.bvh_builder == CRISB_BVH_HOST ||
                d.bvh_builder == CRISB_BVH_DEVICE_WIDE4,
            "scene: unknown bvh_builder");
    if (d.bvh_builder == CRISB_BVH_DEVICE) {
        float max_abs = 0.0f;
        for (float v : s.h_pos) max_abs = std::max(max_abs, std::fabs(v));
        if (build_qbvh_on_device(s, max_abs)) return;
    }
    if (d.bvh_builder != CRISB_BVH_HOST && build_bvh_on_device(s)) return;
    // 4-wide SAH BVH built on the host; triangles stored in leaf order
    WideBvh bvh = build_wide_bvh(s.h_pos.data(), n, kTriLeafMax, kMedianDepth);
    if (bvh.max_stack > kTraversalStack) {
        // a pathological SAH tree: balanced median splits bound the depth
        bvh = build_wide_bvh(s.h_pos.data(), n, kTriLeafMax, 0);
        if (bvh.max_stack > kTraversalStack)
            throw Error(CRISB_ERR_INVALID_ARGUMENT, "scene build: BVH deeper than the traversal stack");
    }
    try {
        validate_wide_bvh(bvh, s.h_pos.data(), n, kTriLeafMax);
    } catch (const std::runtime_error& e) {
        throw Error(CRISB_ERR_INVALID_ARGUMENT, std::string("scene build: ") + e.what());
    }
    s.bvh_max_stack = bvh.max_stack;
    count_children(bvh.nodes, s);
    s.bvh_max_depth = bvh.max_depth;
    s.bvh_on_device = false;
    std::vector<float4> tris(3 * static_cast<size_t>(std::max<uint32_t>(n, 1)), make_float4(0, 0, 0, 0));
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t prim = bvh.order[i];
        const float* p = &s.h_pos[9 * static_cast<size_t>(prim)];
        float pb;
        std::memcpy(&pb, &prim, 4);
        tris[3 * i + 0] = make_float4(p[0], p[1], p[2], 0.0f);
        tris[3 * i + 1] = make_float4(p[3], p[4], p[5], 0.0f);
        tris[3 * i + 2] = make_float4(p[6], p[7], p[8], pb);
    }
    s.tris.upload(tris.data(), tris.size());
    s.nodes.upload(bvh.nodes.data(), bvh.nodes.size());
    check(cudaDeviceSynchronize(), "scene build");
}

void validate_params(const crisb_params& p) {
    require(p.renderer_type >= 0 && p.renderer_type <= 2, "params: renderer_type");
    require(p.max_path_len >= 1 && p.max_path_len <= 255, "params: max_path_len must be in [1, 255]");
    require(p.prefix_len >= 1 && p.prefix_len <= p.max_path_len, "params: prefix_len must be in [1, max_path_len]");
    require(p.prefix_spatial_count >= 0 && p.prefix_spatial_count <= CRISB_MAX_SPATIAL_NEIGH,
            "params: prefix_spatial_count must be in [0, 16]");
    require(p.suffix_spatial_count >= 0 && p.suffix_spatial_count <= CRISB_MAX_SPATIAL_NEIGH,
            "params: suffix_spatial_count must be in [0, 16]");
    require(p.prefix_spatial_rounds >= 0 && p.suffix_spatial_rounds >= 0, "params: negative spatial rounds");
    require(p.gather_n >= 1, "params: gather_n must be >= 1");
    require(p.gather_m >= 1 && p.gather_m <= CRISB_MAX_GATHER_M, "params: gather_m must be in [1, 32]");
    require(p.window_radius >= 0 && p.window_radius < 32768, "params: window_radius");
    require(p.storage == CRISB_STORAGE_FP32 || p.storage == CRISB_STORAGE_FP16, "params: unknown storage");
    require(p.nee_prob >= 0.0f && p.nee_prob <= 1.0f, "params: nee_prob must be in [0, 1]");
    require(p.motion_mode >= CRISB_MOTION_NONE && p.motion_mode <= CRISB_MOTION_REPROJECT, "params: motion_mode");
}

}  // namespace

struct crisb_renderer {
    const crisb_scene* scene = nullptr;
    uint32_t width = 0, height = 0;
    crisb_params params{};
    uint64_t frame_idx = 0, frame_counter = 0;
    uint32_t random = 0;
    int front = 0, back = 0;
    int scur = 0;
    // reservoirs as raw 16-byte words in the layout of params.storage
    DevBuf<uint4> pres[2];
    DevBuf<crisb_prefix_rec> canon_prefix;
    DevBuf<uint4> sres[2];
    DevBuf<uint8_t> nval[2];  // per pixel: usable as a spatial neighbour (same ping-pong as sres)
    DevBuf<crisb_suffix_res_rec> canon_suffix;
    DevBuf<crisb_gbuffer_rec> gbuf;
    DevBuf<crisb_neighbor_rec> neighbors;
    DevBuf<uint32_t> neigh_count;
    DevBuf<float4> entries, knn_leaf;
    DevBuf<uint32_t> pass_status, pass_flags, spatial_nbr, job_items, job_count;
    DevBuf<float4> shift_out, gather_state;
    DevBuf<crisb_suffix_res_rec> gather_cs;
    DevBuf<crisb_prefix_rec> gather_cp;
    DevBuf<float4> gather_ext;          // gatherN > 1 only
    DevBuf<crisb_hit_rec> gather_last;  // gatherN > 1 only
    // The path machines' states and ray queues and the shift machines' job
    // records and ray queues share one allocation: within a pass the path
    // machines finish (the pass's finish kernel reads the last path field, the
    // RNG state) before its shift jobs begin, and the next pass's path
    // machines start after them.
    DevBuf<char> machine_state;
    DevBuf<uint32_t> machine_queue[4];
    DevBuf<uint32_t> wf_count, job_qcount;
    uint32_t slots = 0;
    DevBuf<unsigned int> bounds;
    DevBuf<char> sort_temp;
    LbvhStorage knn;
    DevBuf<int> err;
    cudaStream_t last_stream = nullptr;
    int timing = 0;
    cudaEvent_t ev[7] = {};
    uint32_t launches = 0;
    // statistics level 2: ray, job, node-visit and triangle-test counters,
    // then the resampling kernels' byte tallies
    static constexpr int kRayCounters = 7;
    DevBuf<unsigned long long> ray_count;

    // per-kernel timing: an event after each kernel, tagged with its class
    struct KernelTimer : Marker {
        static constexpr int kMax = 512;
        cudaEvent_t ev[kMax] = {};
        int cls[kMax] = {};
        int n = 0;
        void mark(int c, cudaStream_t st) override {
            if (n >= kMax) return;
            cudaEventRecord(ev[n], st);
            cls[n++] = c;
        }
    } ktimer;

    uint32_t K() const { return static_cast<uint32_t>(params.gather_m - 1); }
    size_t pres_bytes() const {
        return params.storage == CRISB_STORAGE_FP16 ? sizeof(crisb_prefix_res16_rec) : sizeof(crisb_prefix_res_rec);
    }
    size_t sres_bytes() const {
        return params.storage == CRISB_STORAGE_FP16 ? sizeof(crisb_suffix_res16_rec) : sizeof(crisb_suffix_res_rec);
    }
    uint32_t P() const { return width * height; }

    Bufs bufs() const {
        Bufs b;
        const uint32_t f16 = params.storage == CRISB_STORAGE_FP16 ? 1u : 0u;
        b.pres[0] = PresBuf{pres[0].p, f16};
        b.pres[1] = PresBuf{pres[1].p, f16};
        b.canon_prefix = canon_prefix.p;
        b.sres_cur = SresBuf{sres[scur].p, f16};
        b.sres_next = SresBuf{sres[scur ^ 1].p, f16};
        b.nval_cur = nval[scur].p;
        b.nval_next = nval[scur ^ 1].p;
        b.canon_suffix = canon_suffix.p;
        b.gbuf = gbuf.p;
        b.neighbors = neighbors.p;
        b.neigh_count = neigh_count.p;
        b.entries = entries.p;
        b.knn_nodes = knn.nodes.p;
        b.knn_leaf = knn_leaf.p;
        b.knn_pixel = knn.order.p;
        b.knn_n = knn.n.p;
        b.pass_status = pass_status.p;
        b.pass_flags = pass_flags.p;
        b.spatial_nbr = spatial_nbr.p;
        b.job_items = job_items.p;
        b.job_count = job_count.p;
        b.shift_out = shift_out.p;
        b.gather_cs = gather_cs.p;
        b.gather_state = gather_state.p;
        b.gather_ext = params.gather_n > 1 ? gather_ext.p : nullptr;
        b.gather_last = params.gather_n > 1 ? gather_last.p : nullptr;
        b.slots = slots;
        b.job_cap = static_cast<uint32_t>(std::min<size_t>(job_capacity(), 0xFFFFFFFFu));
        b.tally = timing >= 2 && ray_count.p ? ray_count.p + kRayCounters : nullptr;
        b.wf = reinterpret_cast<WfPath*>(machine_state.p);
        for (int q = 0; q < 4; ++q) b.wf_queue[q] = machine_queue[q].p;
        b.wf_count = wf_count.p;
        b.gather_cp = gather_cp.p;
        b.jobs = reinterpret_cast<ShiftJob*>(machine_state.p);
        for (int q = 0; q < 4; ++q) b.job_queue[q] = machine_queue[q].p;
        b.job_qcount = job_qcount.p;
        return b;
    }

    ~crisb_renderer() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        for (auto& e : ktimer.ev)
            if (e) cudaEventDestroy(e);
    }

    Marker* marker() { return timing ? &ktimer : nullptr; }

    // job slots per pixel of the split suffix passes: two shifts per neighbour
    static uint32_t slots_for(const crisb_params& q) {
        const int spatial = std::max(q.suffix_spatial_count, q.prefix_enable_spatial ? q.prefix_spatial_count : 0);
        const uint32_t m = static_cast<uint32_t>(std::max(std::max(q.gather_m - 1, spatial), 1));
        return 2 * m;
    }

    // Shift jobs: the list and the results have a slot for every possible
    // job (4 + 16 bytes); the machines' job records and ray queues (96 bytes
    // a job) hold jobs_per_pixel x P jobs, and a pass's jobs beyond them run
    // in the overflow kernel -- the same results, traced in place.  A 1080p
    // frame of the large workload runs about 2.5 jobs per pixel over all its
    // passes, against 16 slots; a capacity of 1 to 4 jobs per pixel renders
    // it within 1% of the same time.
    // The default (until crisb_set_job_capacity) follows the parameters: 2
    // jobs per pixel, or the prefix spatial pass's 2 per neighbour when that
    // pass runs (RestirPt's spatial reuse lists nearly every neighbour).
    static constexpr uint32_t kDefaultJobsPerPixel = 2;
    uint32_t jobs_per_pixel = kDefaultJobsPerPixel;
    bool jobs_per_pixel_set = false;

    uint32_t effective_jobs_per_pixel() const {
        uint32_t j = jobs_per_pixel;
        if (!jobs_per_pixel_set && params.prefix_enable_spatial)
            j = std::max(j, 2u * static_cast<uint32_t>(std::max(params.prefix_spatial_count, 0)));
        return std::min(j, slots);
    }
    size_t job_capacity() const { return P() * static_cast<size_t>(effective_jobs_per_pixel()); }

    void allocate_jobs() {
        const size_t p = P();
        adjoint_frame = false;  // the resampled-path adjoint reads the frame's shift results
        slots = slots_for(params);
        spatial_nbr.alloc(p * (slots / 2));
        job_items.alloc(p * slots);
        shift_out.alloc(p * slots);
        const size_t state = std::max(p * sizeof(WfPath), job_capacity() * sizeof(ShiftJob));
        machine_state.alloc((state + 255) & ~static_cast<size_t>(255));
        for (int q = 0; q < 4; ++q) machine_queue[q].alloc(std::max(p, job_capacity()));
    }

    void allocate() {
        const uint32_t p = P();
        pass_status.alloc(p);
        pass_flags.alloc(p);
        job_count.alloc(1);
        gather_cs.alloc(p);
        gather_state.alloc(2 * static_cast<size_t>(p));
        gather_cp.alloc(p);
        wf_count.alloc(4);
        check(cudaMemset(wf_count.p, 0, wf_count.bytes()), "memset");
        job_qcount.alloc(4);
        check(cudaMemset(job_qcount.p, 0, job_qcount.bytes()), "memset");
        allocate_jobs();
        for (int i = 0; i < 2; ++i) {
            pres[i].alloc(static_cast<size_t>(p) * (pres_bytes() / 16));
            sres[i].alloc(static_cast<size_t>(p) * (sres_bytes() / 16));
            nval[i].alloc(p);
            check(cudaMemset(nval[i].p, 0, nval[i].bytes()), "memset");
        }
        canon_prefix.alloc(p);
        canon_suffix.alloc(p);
        gbuf.alloc(p);
        neighbors.alloc(static_cast<size_t>(p) * std::max<uint32_t>(K(), 1));
        neigh_count.alloc(p);
        entries.alloc(p);
        knn_leaf.alloc(p);
        bounds.alloc(8);
        knn.alloc(p);
        err.alloc(1);
        check(cudaMemset(err.p, 0, sizeof(int)), "memset");
        check(cudaMemset(neighbors.p, 0, neighbors.bytes()), "memset");
        check(cudaMemset(neigh_count.p, 0, neigh_count.bytes()), "memset");
        const Bufs b0 = bufs();
        k_init_records<<<(p + kPassBlock - 1) / kPassBlock, kPassBlock>>>(b0.pres[0], b0.pres[1], canon_prefix.p,
                                                                         b0.sres_cur, b0.sres_next, canon_suffix.p,
                                                                         gbuf.p, p);
        check(cudaGetLastError(), "init records");
        sort_temp.alloc(rsort::temp_bytes(p));
        check(cudaDeviceSynchronize(), "renderer init");
    }

    void record(int slot, cudaStream_t st) {
        if (timing) check(cudaEventRecord(ev[slot], st), "event");
    }

    // The frame's pass chain as one CUDA graph: the launches are captured on a
    // private stream (nothing runs during capture), the executable graph is
    // updated in place when only kernel parameters changed (camera, frame
    // random, buffer roles) and re-instantiated otherwise, then launched on the
    // caller's stream.  Per-kernel timing records events between launches, so
    // timed frames launch directly.
    bool graph_enabled = true;
    // traversal grid = trace_grid x the blocks resident at once: the queue
    // kernels give each thread a fixed share of rays, and a larger grid evens
    // out the tail (8 measured best on the 1080p workload; crisb_autotune
    // picks it per workload)
    uint32_t trace_grid = 8;
    uint32_t trace_block = 128;  // threads per traversal block
    // views rendering at once as branches of one batch graph: their traversal
    // launches share the GPU, so each takes trace_grid / concurrent_views
    // (at least 1) x the resident blocks (16 views of the multiview workload:
    // 98.6 against 100.0 ms per frame at the full multiplier)
    uint32_t concurrent_views = 1;
    // resampled-path adjoint (crisb_restir_adjoint_*): while enabled, each
    // frame copies the material and emitter tables it renders with (the
    // adjoint's frozen sampling); the last frame's parameters
    bool adjoint_on = false, adjoint_frame = false, has_frame = false;
    DevBuf<crisb_material> frame_mats;
    DevBuf<crisb_emitter> frame_emitters;
    DevBuf<float4> adj_pairs;  // the adjoint's per (pixel, neighbour) scratch
    FrameParams last_fp{};
    // optional sRGB bytes of each frame (ToneMapping after LaunchFrame,
    // src/main.cpp:122-127), written by a last kernel of the frame
    uint8_t* srgb_out = nullptr;
    // temporal reprojection: caller motion vectors, the previous frame's camera
    const float2* motion = nullptr;
    crisb_camera_data prev_cam{};
    bool has_prev_cam = false;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph_exec = nullptr;

    void render(const crisb_camera& cam, float* out, cudaStream_t st) {
        if (!graph_enabled || timing) {
            enqueue(cam, out, st);
            return;
        }
        if (!cap_stream) check(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking), "capture stream");
        check(cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeRelaxed), "begin capture");
        cudaGraph_t g = nullptr;
        try {
            enqueue(cam, out, cap_stream);
        } catch (...) {
            cudaStreamEndCapture(cap_stream, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        check(cudaStreamEndCapture(cap_stream, &g), "end capture");
        if (graph_exec) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(graph_exec, g, &info) != cudaSuccess) {
                cudaGetLastError();
                cudaGraphExecDestroy(graph_exec);
                graph_exec = nullptr;
            }
        }
        if (!graph_exec) {
            const cudaError_t e = cudaGraphInstantiate(&graph_exec, g, 0);
            if (e != cudaSuccess) {
                cudaGraphDestroy(g);
                graph_exec = nullptr;
                check(e, "graph instantiate");
            }
        }
        cudaGraphDestroy(g);
        check(cudaGraphLaunch(graph_exec, st), "graph launch");
        last_stream = st;
    }

    void enqueue(const crisb_camera& cam, float* out, cudaStream_t st) {
        require(out != nullptr, "render_frame: null output");
        launches = 0;
        // Renderer::LaunchFrame (src/Renderer.cpp:211-232)
        ++frame_idx;
        if (cam.changed || !params.enable_accum) frame_idx = 0;
        random = frame_random(params.seed, frame_counter);
        ++frame_counter;
        if (front == 0) {
            front = 1;
            back = 0;
        } else {
            front = 0;
            back = 1;
        }
        FrameParams fp;
        fp.p = params;
        fp.cam = camera_data(cam);
        fp.width = width;
        fp.height = height;
        fp.random = random;
        fp.frame_idx = static_cast<uint32_t>(frame_idx);
        fp.front = front;
        fp.back = back;
        fp.k = K();
        fp.trace_grid = std::max(1u, trace_grid / std::max(1u, concurrent_views));
        // views rendering at once keep shared memory out of their init kernels:
        // the 16-view batch ran 100.7 ms per frame with the staged instances
        // beside 95.7 without, while a single 1080p view gains 0.17 ms from them
        fp.shared_stage = concurrent_views > 1 ? 0u : 1u;
        fp.trace_block = trace_block;
        require(params.motion_mode != CRISB_MOTION_VECTORS || motion != nullptr,
                "render_frame: CRISB_MOTION_VECTORS without motion vectors");
        fp.motion = motion;
        fp.prev_cam = prev_cam;
        fp.has_prev_cam = has_prev_cam ? 1u : 0u;
        prev_cam = fp.cam;
        has_prev_cam = true;
        if (adjoint_on) {
            check(cudaMemcpyAsync(frame_mats.p, scene->mats.p, scene->mats.bytes(), cudaMemcpyDeviceToDevice, st),
                  "adjoint tables");
            check(cudaMemcpyAsync(frame_emitters.p, scene->emitters.p, scene->emitters.bytes(),
                                  cudaMemcpyDeviceToDevice, st),
                  "adjoint tables");
        }
        adjoint_frame = adjoint_on;
        last_fp = fp;
        has_frame = true;
        SceneView s = scene->view(err.p);
        last_stream = st;
        ktimer.n = 0;
        if (timing >= 2) {
            check(cudaMemsetAsync(ray_count.p, 0, (kRayCounters + kTallyKernels) * sizeof(unsigned long long), st),
                  "memset");
            s.ray_count = ray_count.p;
            s.trav_count = ray_count.p + 5;
        }
        Marker* m = marker();
        record(0, st);
        launch_prefix_gen_temp_split(s, fp, bufs(), out, st, m);
        const uint32_t sj = shift_launches_per_phase();
        launches += params.renderer_type == CRISB_RENDERER_PATH_TRACER
                        ? 1
                        : 2 + sj + wf_launches_per_pass(fp, 0) + prefix_pass_extra_launches(fp);
        record(1, st);
        const int type = params.renderer_type;
        if (type == CRISB_RENDERER_PATH_TRACER) {
            tonemap_epilogue(out, st, m);
            for (int i = 2; i < 7; ++i) record(i, st);
            check(cudaGetLastError(), "launch");
            return;
        }
        if (params.prefix_enable_spatial) {
            for (int r = 0; r < params.prefix_spatial_rounds; ++r) {
                launch_prefix_spatial(s, fp, bufs(), out, r, st, m);
                launch_prefix_copy_front_back(fp, bufs(), st);
                if (m) m->mark(kClsOther, st);
                launches += 3 + shift_launches_per_phase();
            }
        }
        record(2, st);
        if (type == CRISB_RENDERER_CONDITIONAL_RESTIR) {
            launch_suffix_gen_temp(s, fp, bufs(), st, m);
            scur ^= 1;
            launches += 2 + sj + wf_launches_per_pass(fp, 1);
            record(3, st);
            if (params.suffix_enable_spatial && params.suffix_spatial_count > 0) {
                for (int r = 0; r < params.suffix_spatial_rounds; ++r) {
                    launch_suffix_spatial(s, fp, bufs(), st, m);
                    launches += 2 + sj;
                    scur ^= 1;
                }
            }
            record(4, st);
            lbvh::Work w = knn.work(err.p);
            launch_store_entries(s, fp, bufs(), w, bounds.p, st);
            check(rsort::sort_high32(knn.keys_in.p, knn.keys.p, sort_temp.p, sort_temp.bytes(), P(), st),
                  "radix sort");
            launch_knn_finish(fp, bufs(), w, knn_leaf.p, st);
            if (m) m->mark(kClsSearch, st);
            launches += 3 + 4 + rsort::kLaunches;
            record(5, st);
            if (params.gather_n > 1 && !gather_ext.p) {
                gather_ext.alloc(3 * static_cast<size_t>(P()));
                gather_last.alloc(P());
            }
            launch_final_gather_split(s, fp, bufs(), out, st, m);
            launches += 3 + sj + wf_launches_per_pass(fp, 2);
            if (params.gather_n > 1)
                launches += 1 + static_cast<uint32_t>(params.gather_n - 1) * (3 + sj);
        } else {
            record(3, st);
            record(4, st);
            record(5, st);
        }
        tonemap_epilogue(out, st, m);
        record(6, st);
        check(cudaGetLastError(), "launch");
    }

    void tonemap_epilogue(const float* out, cudaStream_t st, Marker* m) {
        if (!srgb_out) return;
        check(launch_tonemap_srgb8(out, srgb_out, width * height, st), "tonemap");
        if (m) m->mark(kClsOther, st);
        ++launches;
    }
};

namespace {

// Times candidate settings of one knob on renderer t: every candidate renders
// `frames` frames of `cam`, interleaved frame by frame so that drift hits all
// of them alike, after one untimed frame each (graph instantiation per shape).
// Returns the per-candidate total milliseconds.
template <class Apply>
std::vector<float> time_candidates(crisb_renderer& t, const crisb_camera& cam, float* out, cudaStream_t st,
                                   uint32_t frames, size_t count, Apply apply) {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    check(cudaEventCreate(&e0), "event");
    check(cudaEventCreate(&e1), "event");
    std::vector<float> total(count, 0.0f);
    for (size_t k = 0; k < count; ++k) {
        apply(k);
        t.render(cam, out, st);
    }
    for (uint32_t f = 0; f < std::max<uint32_t>(frames, 3); ++f) {
        for (size_t k = 0; k < count; ++k) {
            apply(k);
            check(cudaEventRecord(e0, st), "event");
            t.render(cam, out, st);
            check(cudaEventRecord(e1, st), "event");
            check(cudaEventSynchronize(e1), "sync");
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
            total[k] += ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return total;
}

size_t fastest(const std::vector<float>& v) { return static_cast<size_t>(std::min_element(v.begin(), v.end()) - v.begin()); }

}  // namespace

extern "C" {

const char* crisb_version(void) { return "crisb 0.1.0 (sm_100a)"; }

int crisb_last_error(char* buf, size_t len) {
    if (!buf || len == 0) return CRISB_ERR_INVALID_ARGUMENT;
    std::strncpy(buf, g_last_error.c_str(), len - 1);
    buf[len - 1] = 0;
    return CRISB_OK;
}

int crisb_params_default(crisb_params* out, float scene_size) {
    return guarded([&] {
        require(out != nullptr, "null params");
        std::memset(out, 0, sizeof(*out));
        // Renderer::Renderer, src/Renderer.cpp:34-58
        out->renderer_type = CRISB_RENDERER_PATH_TRACER;
        out->nee_prob = 0.3f;
        out->max_path_len = 8;
        out->enable_accum = 0;
        out->recon_min_distance = 0.01f * scene_size;
        out->recon_min_roughness = 0.2f;
        out->prefix_len = 2;
        out->prefix_enable_temporal = 1;
        out->prefix_enable_spatial = 0;
        out->prefix_spatial_count = 1;
        out->prefix_spatial_rounds = 1;
        out->suffix_enable_temporal = 1;
        out->suffix_enable_spatial = 1;
        out->suffix_spatial_count = 1;
        out->suffix_spatial_rounds = 1;
        out->gather_n = 1;
        out->gather_m = 1;
        out->gather_radius = 0.01f;
        out->gather_radius_type = CRISB_RADIUS_PATH_LENGTH;
        out->window_radius = 10;
        out->storage = CRISB_STORAGE_FP32;
        out->seed = 0;
    });
}

int crisb_camera_get_data(const crisb_camera* cam, crisb_camera_data* out) {
    return guarded([&] {
        require(cam && out, "null argument");
        *out = camera_data(*cam);
    });
}

int crisb_scene_create(const crisb_scene_desc* desc, crisb_scene** out) {
    return guarded([&] {
        require(desc && out, "null argument");
        *out = nullptr;
        auto s = std::make_unique<crisb_scene>();
        build_scene(*desc, *s);
        *out = s.release();
    });
}

int crisb_scene_destroy(crisb_scene* scene) {
    delete scene;
    return CRISB_OK;
}

int crisb_scene_size(const crisb_scene* scene, float* out) {
    return guarded([&] {
        require(scene && out, "null argument");
        *out = scene->scene_size;
    });
}

int crisb_scene_num_triangles(const crisb_scene* scene, uint32_t* out) {
    return guarded([&] {
        require(scene && out, "null argument");
        *out = scene->num_tris;
    });
}

int crisb_scene_bvh_info(const crisb_scene* scene, crisb_bvh_info* out) {
    return guarded([&] {
        require(scene && out, "null argument");
        const bool q = scene->qnodes.p != nullptr;
        out->format = q ? CRISB_BVH_FORMAT_COMPRESSED8 : CRISB_BVH_FORMAT_WIDE4;
        out->on_device = scene->bvh_on_device ? 1u : 0u;
        out->num_nodes = static_cast<uint32_t>(q ? scene->qnodes.n : scene->nodes.n);
        out->node_bytes = q ? static_cast<uint32_t>(sizeof(Bvh8QNode)) : static_cast<uint32_t>(sizeof(Bvh4Node));
        out->stack_bound = scene->bvh_max_stack;
        out->depth = scene->bvh_max_depth;
        out->inner_children = scene->bvh_inner_children;
        out->leaf_children = scene->bvh_leaf_children;
    });
}

int crisb_scene_read_triangles(const crisb_scene* scene, float* positions, float* normals, uint32_t* materials) {
    return guarded([&] {
        require(scene != nullptr, "null scene");
        if (positions) std::memcpy(positions, scene->h_pos.data(), scene->h_pos.size() * 4);
        if (normals) std::memcpy(normals, scene->h_nrm.data(), scene->h_nrm.size() * 4);
        if (materials) std::memcpy(materials, scene->h_mat.data(), scene->h_mat.size() * 4);
    });
}

int crisb_trace_rays(const crisb_scene* scene, const float* rays_dev, crisb_trace_hit* hits_dev, uint32_t n,
                     int any_hit, void* stream) {
    return guarded([&] {
        require(scene && rays_dev && hits_dev, "null argument");
        if (n == 0) return;
        const SceneView s = scene->view(scene->err.p);
        k_trace_rays<<<(n + kPassBlock - 1) / kPassBlock, kPassBlock, 0, static_cast<cudaStream_t>(stream)>>>(
            s, rays_dev, hits_dev, n, any_hit);
        check(cudaGetLastError(), "k_trace_rays");
    });
}

int crisb_renderer_create(const crisb_scene* scene, uint32_t width, uint32_t height, const crisb_params* params,
                          crisb_renderer** out) {
    return guarded([&] {
        require(scene && params && out, "null argument");
        *out = nullptr;
        require(width > 0 && height > 0 && width < 65536 && height < 65536, "renderer: bad resolution");
        require(static_cast<uint64_t>(width) * height < (1ull << 26), "renderer: too many pixels (max 2^26)");
        validate_params(*params);
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        require(dev == scene->device, "renderer: scene lives on another device");
        auto r = std::make_unique<crisb_renderer>();
        r->scene = scene;
        r->width = width;
        r->height = height;
        r->params = *params;
        r->allocate();
        *out = r.release();
    });
}

int crisb_renderer_destroy(crisb_renderer* r) {
    delete r;
    return CRISB_OK;
}

}  // extern "C"

// Several renderers (views) whose frames run as parallel branches of one CUDA
// graph: the captured launches of every view hang off one fork event and join
// before the graph ends, so small views and the tails of large ones overlap
// on the device instead of running one view after another.
struct crisb_batch {
    std::vector<crisb_renderer*> views;
    cudaStream_t cap = nullptr;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> done;
    cudaEvent_t fork = nullptr;
    cudaGraphExec_t exec = nullptr;

    ~crisb_batch() {
        if (exec) cudaGraphExecDestroy(exec);
        for (auto& e : done)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        for (auto& s : branch)
            if (s) cudaStreamDestroy(s);
        if (cap) cudaStreamDestroy(cap);
    }

    void render(const crisb_camera* cams, float* const* outs, cudaStream_t st) {
        for (size_t k = 0; k < views.size(); ++k) {
            require(outs[k] != nullptr, "batch: null output");
            require(views[k]->timing == 0, "batch: per-kernel timing must be off for batched frames");
        }
        check(cudaStreamBeginCapture(cap, cudaStreamCaptureModeRelaxed), "begin capture");
        cudaGraph_t g = nullptr;
        try {
            check(cudaEventRecord(fork, cap), "fork");
            for (size_t k = 0; k < views.size(); ++k) {
                check(cudaStreamWaitEvent(branch[k], fork, 0), "branch wait");
                views[k]->concurrent_views = static_cast<uint32_t>(views.size());
                views[k]->enqueue(cams[k], outs[k], branch[k]);
                views[k]->concurrent_views = 1;
                check(cudaEventRecord(done[k], branch[k]), "join");
                check(cudaStreamWaitEvent(cap, done[k], 0), "join wait");
            }
        } catch (...) {
            for (auto* v : views) v->concurrent_views = 1;
            cudaStreamEndCapture(cap, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        check(cudaStreamEndCapture(cap, &g), "end capture");
        if (exec) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(exec, g, &info) != cudaSuccess) {
                cudaGetLastError();
                cudaGraphExecDestroy(exec);
                exec = nullptr;
            }
        }
        if (!exec) {
            const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
            if (e != cudaSuccess) {
                cudaGraphDestroy(g);
                exec = nullptr;
                check(e, "graph instantiate");
            }
        }
        cudaGraphDestroy(g);
        check(cudaGraphLaunch(exec, st), "graph launch");
        for (auto* v : views) v->last_stream = st;
    }
};

extern "C" {

int crisb_scene_get_materials(const crisb_scene* scene, crisb_material* out, uint32_t n) {
    return guarded([&] {
        require(scene && out, "null argument");
        require(n == scene->mats.n, "scene: material count mismatch");
        check(cudaMemcpy(out, scene->mats.p, n * sizeof(crisb_material), cudaMemcpyDeviceToHost), "read");
    });
}

int crisb_scene_set_materials(crisb_scene* scene, const crisb_material* mats, uint32_t n) {
    return guarded([&] {
        require(scene && mats, "null argument");
        require(n == scene->mats.n, "scene: material count mismatch");
        check(cudaDeviceSynchronize(), "sync");
        check(cudaMemcpy(scene->mats.p, mats, n * sizeof(crisb_material), cudaMemcpyHostToDevice), "write");
    });
}

int crisb_scene_set_emitter_colors(crisb_scene* scene, const float* rgb, uint32_t n) {
    return guarded([&] {
        require(scene && rgb, "null argument");
        require(n == scene->num_emitters, "scene: emitter count mismatch");
        std::vector<crisb_emitter> e(n);
        check(cudaDeviceSynchronize(), "sync");
        check(cudaMemcpy(e.data(), scene->emitters.p, n * sizeof(crisb_emitter), cudaMemcpyDeviceToHost), "read");
        for (uint32_t k = 0; k < n; ++k)
            for (int c = 0; c < 3; ++c) e[k].color[c] = rgb[3 * k + c];
        check(cudaMemcpy(scene->emitters.p, e.data(), n * sizeof(crisb_emitter), cudaMemcpyHostToDevice), "write");
    });
}

int crisb_batch_create(crisb_renderer* const* renderers, uint32_t n, crisb_batch** out) {
    return guarded([&] {
        require(renderers && out && n > 0, "batch: null argument or no renderers");
        *out = nullptr;
        auto b = std::make_unique<crisb_batch>();
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        for (uint32_t k = 0; k < n; ++k) {
            require(renderers[k] != nullptr, "batch: null renderer");
            require(renderers[k]->scene->device == dev, "batch: renderer on another device");
            for (uint32_t j = 0; j < k; ++j) require(renderers[j] != renderers[k], "batch: renderer listed twice");
            b->views.push_back(renderers[k]);
        }
        check(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking), "stream");
        b->branch.assign(n, nullptr);
        b->done.assign(n, nullptr);
        for (uint32_t k = 0; k < n; ++k) {
            check(cudaStreamCreateWithFlags(&b->branch[k], cudaStreamNonBlocking), "stream");
            check(cudaEventCreateWithFlags(&b->done[k], cudaEventDisableTiming), "event");
        }
        check(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "event");
        *out = b.release();
    });
}

}  // extern "C"

struct crisb_adjoint {
    crisb_scene* scene = nullptr;
    uint32_t width = 0, height = 0;
    crisb_params params{};
    DevBuf<crisb_material> sample_mats;  // theta0

    FrameParams frame(const crisb_camera& cam, uint64_t index) const {
        FrameParams fp;
        std::memset(&fp, 0, sizeof(fp));
        fp.p = params;
        fp.cam = camera_data(cam);
        fp.width = width;
        fp.height = height;
        fp.random = frame_random(params.seed, index);
        fp.k = 0;
        return fp;
    }
    void freeze() {
        sample_mats.alloc(scene->mats.n);
        check(cudaMemcpy(sample_mats.p, scene->mats.p, scene->mats.bytes(), cudaMemcpyDeviceToDevice), "freeze");
        check(cudaDeviceSynchronize(), "freeze");
    }
};

extern "C" {

int crisb_adjoint_create(crisb_scene* scene, uint32_t width, uint32_t height, const crisb_params* params,
                         crisb_adjoint** out) {
    return guarded([&] {
        require(scene && params && out, "null argument");
        *out = nullptr;
        require(width > 0 && height > 0 && static_cast<uint64_t>(width) * height < (1ull << 26), "adjoint: bad size");
        validate_params(*params);
        require(params->max_path_len <= 16, "adjoint: max_path_len must be <= 16");
        require(scene->num_emitters > 0, "adjoint: the scene has no emitters");
        require(!scene->textured, "adjoint: textured materials are not differentiated");
        auto a = std::make_unique<crisb_adjoint>();
        a->scene = scene;
        a->width = width;
        a->height = height;
        a->params = *params;
        a->freeze();
        *out = a.release();
    });
}

int crisb_adjoint_destroy(crisb_adjoint* a) {
    delete a;
    return CRISB_OK;
}

int crisb_adjoint_refreeze(crisb_adjoint* a) {
    return guarded([&] {
        require(a != nullptr, "null argument");
        a->freeze();
    });
}

int crisb_adjoint_forward(crisb_adjoint* a, const crisb_camera* cam, uint64_t frame, float* out_rgb_dev,
                          void* stream) {
    return guarded([&] {
        require(a && cam && out_rgb_dev, "null argument");
        const FrameParams fp = a->frame(*cam, frame);
        const SceneView s = a->scene->view(a->scene->err.p);
        adjoint_forward(s, a->sample_mats.p, static_cast<uint32_t>(a->sample_mats.n), fp, out_rgb_dev,
                        static_cast<cudaStream_t>(stream));
        check(cudaGetLastError(), "adjoint forward");
    });
}

int crisb_adjoint_backward(crisb_adjoint* a, const crisb_camera* cam, uint64_t frame, const float* d_image_dev,
                           float* d_materials_dev, float* d_emitters_dev, void* stream) {
    return guarded([&] {
        require(a && cam && d_image_dev && d_materials_dev && d_emitters_dev, "null argument");
        const FrameParams fp = a->frame(*cam, frame);
        const SceneView s = a->scene->view(a->scene->err.p);
        adjoint_backward(s, a->sample_mats.p, static_cast<uint32_t>(a->sample_mats.n), fp, d_image_dev,
                         d_materials_dev, d_emitters_dev, static_cast<cudaStream_t>(stream));
        check(cudaGetLastError(), "adjoint backward");
    });
}

int crisb_batch_destroy(crisb_batch* b) {
    delete b;
    return CRISB_OK;
}

int crisb_batch_render(crisb_batch* b, const crisb_camera* cams, float* const* outs, void* stream) {
    return guarded([&] {
        require(b && cams && outs, "null argument");
        b->render(cams, outs, static_cast<cudaStream_t>(stream));
    });
}

int crisb_renderer_set_params(crisb_renderer* r, const crisb_params* params) {
    return guarded([&] {
        require(r && params, "null argument");
        validate_params(*params);
        require(params->storage == r->params.storage, "params: storage is fixed when the renderer is created");
        const bool realloc_neighbors = params->gather_m != r->params.gather_m;
        const size_t cap_before = r->job_capacity();
        const uint32_t slots_before = r->slots;
        r->params = *params;
        r->slots = crisb_renderer::slots_for(*params);
        const bool realloc_jobs = r->slots != slots_before || r->job_capacity() != cap_before;
        r->slots = slots_before;
        if (realloc_neighbors || realloc_jobs) check(cudaDeviceSynchronize(), "sync");
        if (realloc_neighbors) {
            r->adjoint_frame = false;  // the frame's neighbour lists are gone
            r->neighbors.alloc(static_cast<size_t>(r->P()) * std::max<uint32_t>(r->K(), 1));
            check(cudaMemset(r->neighbors.p, 0, r->neighbors.bytes()), "memset");
        }
        if (realloc_jobs) r->allocate_jobs();
    });
}

int crisb_renderer_get_params(const crisb_renderer* r, crisb_params* out) {
    return guarded([&] {
        require(r && out, "null argument");
        *out = r->params;
    });
}

int crisb_render_frame(crisb_renderer* r, const crisb_camera* cam, float* out_rgb_dev, void* stream) {
    return guarded([&] {
        require(r && cam, "null argument");
        r->render(*cam, out_rgb_dev, static_cast<cudaStream_t>(stream));
    });
}

int crisb_restir_adjoint_enable(crisb_renderer* r, int on) {
    return guarded([&] {
        require(r != nullptr, "null renderer");
        if (on && r->frame_mats.n != r->scene->mats.n) r->frame_mats.alloc(r->scene->mats.n);
        if (on && r->frame_emitters.n != r->scene->emitters.n) r->frame_emitters.alloc(r->scene->emitters.n);
        r->adjoint_on = on != 0;
    });
}

namespace {
void restir_adjoint_check(const crisb_renderer* r) {
    require(r->has_frame && r->adjoint_frame,
            "restir adjoint: enable it (crisb_restir_adjoint_enable) and render a frame first (a parameter or "
            "job-capacity change that reallocated the frame's buffers ends its adjoint)");
    const crisb_params& p = r->last_fp.p;  // the frame's parameters
    require(p.renderer_type == CRISB_RENDERER_CONDITIONAL_RESTIR, "restir adjoint: Conditional ReSTIR only");
    require(p.gather_n == 1, "restir adjoint: gather_n must be 1");
    require(p.storage == CRISB_STORAGE_FP32, "restir adjoint: FP32 reservoir storage only");
    require(p.max_path_len <= 16, "restir adjoint: max_path_len must be <= 16");
    require(!r->scene->textured, "restir adjoint: textured materials are not differentiated");
    require(r->scene->num_emitters > 0, "restir adjoint: the scene has no emitters");
    require(r->frame_mats.n == r->scene->mats.n && r->frame_emitters.n == r->scene->emitters.n,
            "restir adjoint: table sizes changed");
}
float4* restir_adjoint_pairs(crisb_renderer* r) {
    const size_t need = static_cast<size_t>(r->last_fp.width) * r->last_fp.height * std::max(1u, r->last_fp.k);
    if (r->adj_pairs.n < need) r->adj_pairs.alloc(need);
    return r->adj_pairs.p;
}
}  // namespace

int crisb_restir_adjoint_forward(crisb_renderer* r, float* out_rgb_dev, void* stream) {
    return guarded([&] {
        require(r && out_rgb_dev, "null argument");
        restir_adjoint_check(r);
        restir_adjoint_forward(r->scene->view(r->err.p), r->frame_mats.p, r->frame_emitters.p,
                               static_cast<uint32_t>(r->scene->mats.n), r->last_fp, r->bufs(), restir_adjoint_pairs(r),
                               out_rgb_dev, static_cast<cudaStream_t>(stream));
        check(cudaGetLastError(), "restir adjoint forward");
    });
}

int crisb_restir_adjoint_backward(crisb_renderer* r, const float* d_image_dev, float* d_materials_dev,
                                  float* d_emitters_dev, void* stream) {
    return guarded([&] {
        require(r && d_image_dev && d_materials_dev && d_emitters_dev, "null argument");
        restir_adjoint_check(r);
        restir_adjoint_backward(r->scene->view(r->err.p), r->frame_mats.p, r->frame_emitters.p,
                                static_cast<uint32_t>(r->scene->mats.n), r->last_fp, r->bufs(), restir_adjoint_pairs(r),
                                d_image_dev, d_materials_dev, d_emitters_dev, static_cast<cudaStream_t>(stream));
        check(cudaGetLastError(), "restir adjoint backward");
    });
}

int crisb_tonemap_srgb8(const float* rgb_dev, uint8_t* srgb_dev, uint32_t num_pixels, void* stream) {
    return guarded([&] {
        if (num_pixels == 0) return;  // nothing is read or written
        require(rgb_dev && srgb_dev, "null argument");
        check(launch_tonemap_srgb8(rgb_dev, srgb_dev, num_pixels, static_cast<cudaStream_t>(stream)), "tonemap");
    });
}

int crisb_set_motion_vectors(crisb_renderer* r, const float* motion_dev) {
    return guarded([&] {
        require(r != nullptr, "null renderer");
        require(reinterpret_cast<uintptr_t>(motion_dev) % alignof(float2) == 0, "motion vectors: 8-byte alignment");
        r->motion = reinterpret_cast<const float2*>(motion_dev);
    });
}

int crisb_set_srgb_output(crisb_renderer* r, uint8_t* srgb_dev) {
    return guarded([&] {
        require(r != nullptr, "null renderer");
        r->srgb_out = srgb_dev;
    });
}

int crisb_srgb8_thresholds(float* thresholds, float* c_max) {
    return guarded([&] {
        require(thresholds && c_max, "null argument");
        srgb8_thresholds(thresholds, c_max);
    });
}

int crisb_set_trace_grid(crisb_renderer* r, uint32_t blocks_per_resident_block) {
    return guarded([&] {
        require(r != nullptr, "null renderer");
        require(blocks_per_resident_block >= 1 && blocks_per_resident_block <= 64, "trace grid must be in [1, 64]");
        r->trace_grid = blocks_per_resident_block;
    });
}

int crisb_autotune_ex(crisb_renderer* r, const crisb_camera* cam, uint32_t frames, crisb_tuning* out) {
    return guarded([&] {
        require(r && cam && frames > 0, "autotune: null argument or no frames");
        // a scratch renderer of the same scene, size and parameters: the
        // caller's renderer keeps its state
        crisb_renderer* t = nullptr;
        if (crisb_renderer_create(r->scene, r->width, r->height, &r->params, &t) != CRISB_OK)
            throw Error(CRISB_ERR_CUDA, g_last_error);
        std::unique_ptr<crisb_renderer> tmp(t);
        DevBuf<float> buf;
        buf.alloc(static_cast<size_t>(r->P()) * 3);
        cudaStream_t st = nullptr;
        check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
        // warm up until the reservoirs carry history (the per-frame cost of a
        // fresh renderer's first frames is lower)
        for (int f = 0; f < 4; ++f) tmp->render(*cam, buf.p, st);
        // coordinate descent: traversal block size, traversal grid, then the
        // shift machines' job capacity (the smallest within 1% of the fastest:
        // capacity costs memory, 96 bytes per job)
        const uint32_t blocks[] = {64, 128, 256};
        auto tb = time_candidates(*tmp, *cam, buf.p, st, frames, 3, [&](size_t k) { tmp->trace_block = blocks[k]; });
        tmp->trace_block = blocks[fastest(tb)];
        const uint32_t grids[] = {1, 2, 4, 8, 16};
        auto tg = time_candidates(*tmp, *cam, buf.p, st, frames, 5, [&](size_t k) { tmp->trace_grid = grids[k]; });
        tmp->trace_grid = grids[fastest(tg)];
        std::vector<uint32_t> caps;
        for (uint32_t c : {1u, 2u, 4u, 8u})
            if (c <= tmp->slots) caps.push_back(c);
        if (caps.empty() || caps.back() != tmp->slots) caps.push_back(tmp->slots);
        const uint32_t base_cap = tmp->jobs_per_pixel;
        auto tc = time_candidates(*tmp, *cam, buf.p, st, frames, caps.size(), [&](size_t k) {
            if (tmp->jobs_per_pixel == caps[k]) return;
            check(cudaStreamSynchronize(st), "sync");
            tmp->jobs_per_pixel = caps[k];
            tmp->jobs_per_pixel_set = true;
            tmp->allocate_jobs();
        });
        const float best_cap_ms = tc[fastest(tc)];
        uint32_t cap = caps.back();
        for (size_t k = 0; k < caps.size(); ++k)
            if (tc[k] <= 1.01f * best_cap_ms) {
                cap = caps[k];
                break;
            }
        (void)base_cap;
        check(cudaStreamSynchronize(st), "sync");
        cudaStreamDestroy(st);
        r->trace_block = tmp->trace_block;
        r->trace_grid = tmp->trace_grid;
        if (r->effective_jobs_per_pixel() != std::min(cap, r->slots) || !r->jobs_per_pixel_set) {
            check(cudaDeviceSynchronize(), "job capacity");
            r->jobs_per_pixel = cap;
            r->jobs_per_pixel_set = true;
            r->allocate_jobs();
        }
        if (out) {
            out->trace_block = r->trace_block;
            out->trace_grid = r->trace_grid;
            out->jobs_per_pixel = std::min(cap, r->slots);
            out->frame_ms = std::min(tb[fastest(tb)], std::min(tg[fastest(tg)], best_cap_ms)) /
                            static_cast<float>(std::max<uint32_t>(frames, 3));
        }
    });
}

int crisb_autotune_spatial(crisb_renderer* r, const crisb_camera* cam, uint32_t frames, float budget_ms,
                           uint32_t* chosen, float* chosen_ms) {
    return guarded([&] {
        require(r && cam && frames > 0 && budget_ms > 0.0f, "autotune spatial: null argument, no frames or no budget");
        require(r->params.renderer_type == CRISB_RENDERER_CONDITIONAL_RESTIR && r->params.suffix_enable_spatial &&
                    r->params.suffix_spatial_rounds > 0,
                "autotune spatial: Conditional ReSTIR with suffix spatial reuse only");
        DevBuf<float> buf;
        buf.alloc(static_cast<size_t>(r->P()) * 3);
        cudaStream_t st = nullptr;
        check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
        // ascending: the frame time grows with the count, so the first count
        // over the budget ends the search
        const uint32_t counts[] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16};
        uint32_t best = 0;
        float best_ms = 0.0f, first_ms = 0.0f;
        for (uint32_t c : counts) {
            if (c > CRISB_MAX_SPATIAL_NEIGH) break;
            crisb_params p = r->params;
            p.suffix_spatial_count = static_cast<int>(c);
            // a scratch renderer with the caller's launch settings; the
            // caller's reservoirs are left alone
            crisb_renderer* t = nullptr;
            if (crisb_renderer_create(r->scene, r->width, r->height, &p, &t) != CRISB_OK)
                throw Error(CRISB_ERR_CUDA, g_last_error);
            std::unique_ptr<crisb_renderer> tmp(t);
            tmp->trace_block = r->trace_block;
            tmp->trace_grid = r->trace_grid;
            if (r->jobs_per_pixel_set) {
                tmp->jobs_per_pixel = r->jobs_per_pixel;
                tmp->jobs_per_pixel_set = true;
                tmp->allocate_jobs();
            }
            for (int f = 0; f < 4; ++f) tmp->render(*cam, buf.p, st);  // reservoirs with history
            check(cudaEventRecord(e0, st), "event");
            for (uint32_t f = 0; f < frames; ++f) tmp->render(*cam, buf.p, st);
            check(cudaEventRecord(e1, st), "event");
            check(cudaEventSynchronize(e1), "sync");
            float ms = 0.0f;
            check(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
            ms /= static_cast<float>(frames);
            if (c == counts[0]) first_ms = ms;
            if (ms > budget_ms) break;
            best = c;
            best_ms = ms;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        check(cudaStreamSynchronize(st), "sync");
        cudaStreamDestroy(st);
        if (best == 0) {  // nothing fits: the cheapest
            best = counts[0];
            best_ms = first_ms;
        }
        crisb_params p = r->params;
        p.suffix_spatial_count = static_cast<int>(best);
        if (crisb_renderer_set_params(r, &p) != CRISB_OK) throw Error(CRISB_ERR_INVALID_ARGUMENT, g_last_error);
        if (chosen) *chosen = best;
        if (chosen_ms) *chosen_ms = best_ms;
    });
}

int crisb_autotune(crisb_renderer* r, const crisb_camera* cam, uint32_t frames, uint32_t* chosen) {
    crisb_tuning t{};
    const int rc = crisb_autotune_ex(r, cam, frames, &t);
    if (rc == CRISB_OK && chosen) *chosen = t.trace_grid;
    return rc;
}

int crisb_set_trace_block(crisb_renderer* r, uint32_t threads) {
    return guarded([&] {
        require(r != nullptr, "null renderer");
        require(threads == 64 || threads == 128 || threads == 256, "trace block: 64, 128 or 256 threads");
        r->trace_block = threads;
    });
}

int crisb_set_graph(crisb_renderer* r, int enable) {
    return guarded([&] {
        require(r != nullptr, "null renderer");
        r->graph_enabled = enable != 0;
    });
}

int crisb_frame_index(const crisb_renderer* r, uint64_t* out) {
    return guarded([&] {
        require(r && out, "null argument");
        *out = r->frame_idx;
    });
}

int crisb_frame_random(const crisb_renderer* r, uint32_t* out) {
    return guarded([&] {
        require(r && out, "null argument");
        *out = r->random;
    });
}

int crisb_set_job_capacity(crisb_renderer* r, uint32_t jobs_per_pixel) {
    return guarded([&] {
        require(r != nullptr, "null renderer");
        require(jobs_per_pixel <= CRISB_MAX_GATHER_M * 2, "job capacity: at most 64 jobs per pixel");
        r->jobs_per_pixel_set = true;
        if (jobs_per_pixel == r->jobs_per_pixel && r->job_capacity() == r->P() * static_cast<size_t>(
                                                                                std::min(jobs_per_pixel, r->slots)))
            return;
        check(cudaDeviceSynchronize(), "job capacity");
        r->jobs_per_pixel = jobs_per_pixel;
        r->allocate_jobs();
    });
}

int crisb_get_job_capacity(const crisb_renderer* r, uint32_t* jobs_per_pixel) {
    return guarded([&] {
        require(r && jobs_per_pixel, "null argument");
        *jobs_per_pixel = r->effective_jobs_per_pixel();
    });
}

int crisb_set_timing(crisb_renderer* r, int enable) {
    return guarded([&] {
        require(r != nullptr, "null renderer");
        require(enable >= 0 && enable <= 2, "timing level must be 0, 1 or 2");
        if (enable && !r->ev[0]) {
            for (auto& e : r->ev) check(cudaEventCreate(&e), "event create");
            for (auto& e : r->ktimer.ev) check(cudaEventCreate(&e), "event create");
        }
        if (enable >= 2 && !r->ray_count.p) r->ray_count.alloc(crisb_renderer::kRayCounters + kTallyKernels);
        r->timing = enable;
    });
}

int crisb_get_stats(crisb_renderer* r, crisb_stats* out) {
    return guarded([&] {
        require(r && out, "null argument");
        std::memset(out, 0, sizeof(*out));
        out->kernel_launches = r->launches;
        if (!r->timing) return;
        check(cudaEventSynchronize(r->ev[6]), "event sync");
        float ms[6];
        for (int i = 0; i < 6; ++i) check(cudaEventElapsedTime(&ms[i], r->ev[i], r->ev[i + 1]), "elapsed");
        out->prefix_gen_temp_ms = ms[0];
        out->prefix_spatial_ms = ms[1];
        out->suffix_gen_temp_ms = ms[2];
        out->suffix_spatial_ms = ms[3];
        out->prefix_store_ms = ms[4];
        out->final_gather_ms = ms[5];
        check(cudaEventElapsedTime(&out->total_ms, r->ev[0], r->ev[6]), "elapsed");
        float cls_ms[6] = {0, 0, 0, 0, 0, 0};
        cudaEvent_t prev = r->ev[0];
        for (int j = 0; j < r->ktimer.n; ++j) {
            float t = 0.0f;
            check(cudaEventElapsedTime(&t, prev, r->ktimer.ev[j]), "elapsed");
            cls_ms[r->ktimer.cls[j]] += t;
            prev = r->ktimer.ev[j];
        }
        out->trace_ms = cls_ms[kClsTrace];
        out->shift_ms = cls_ms[kClsShift];
        out->resample_ms = cls_ms[kClsResample];
        out->search_ms = cls_ms[kClsSearch];
        out->shade_ms = cls_ms[kClsShade];
        out->other_ms = cls_ms[kClsOther];
        if (r->timing >= 2) {
            constexpr int kRayCounters = crisb_renderer::kRayCounters;
            unsigned long long rc[kRayCounters + kTallyKernels] = {};
            check(cudaMemcpy(rc, r->ray_count.p, sizeof(rc), cudaMemcpyDeviceToHost), "ray counters");
            for (int k = 0; k < kTallyKernels; ++k) out->resample_bytes[k] = rc[kRayCounters + k];
            out->closest_rays = rc[0] + rc[2];
            out->shadow_rays = rc[1] + rc[3];
            out->shift_closest_rays = rc[2];
            out->shift_shadow_rays = rc[3];
            out->shift_jobs = rc[4];
            out->node_visits = rc[5];
            out->tri_tests = rc[6];
        }
    });
}

int crisb_check_device_errors(crisb_renderer* r) {
    int code = CRISB_OK;
    const int st = guarded([&] {
        require(r != nullptr, "null renderer");
        check(cudaStreamSynchronize(r->last_stream), "stream sync");
        int e = 0;
        check(cudaMemcpy(&e, r->err.p, 4, cudaMemcpyDeviceToHost), "read error word");
        if (e) {
            g_last_error = "device error word " + std::to_string(e) +
                           ((e & kDevErrStack) ? " (traversal stack overflow)" : "") +
                           ((e & kDevErrIterations) ? " (traversal iteration cap)" : "") +
                           ((e & kDevErrKnn) ? " (endpoint search cap)" : "");
            code = CRISB_ERR_DEVICE_FAULT;
        }
    });
    return st != CRISB_OK ? st : code;
}

int crisb_debug_size(const crisb_renderer* r, int id, size_t* out) {
    return guarded([&] {
        require(r && out, "null argument");
        const size_t P = r->P();
        switch (id) {
            case CRISB_BUF_PREFIX_RES_FRONT:
            case CRISB_BUF_PREFIX_RES_BACK: *out = P * r->pres_bytes(); break;
            case CRISB_BUF_CANON_PREFIX: *out = P * sizeof(crisb_prefix_rec); break;
            case CRISB_BUF_SUFFIX_RES_FRONT:
            case CRISB_BUF_SUFFIX_RES_BACK: *out = P * r->sres_bytes(); break;
            case CRISB_BUF_CANON_SUFFIX: *out = P * sizeof(crisb_suffix_rec); break;
            case CRISB_BUF_GBUFFER: *out = P * sizeof(crisb_gbuffer_rec); break;
            case CRISB_BUF_NEIGHBORS: *out = P * r->K() * sizeof(crisb_neighbor_rec); break;
            case CRISB_BUF_NEIGHBOR_COUNT: *out = P * sizeof(uint32_t); break;
            default: require(false, "debug: unknown buffer id");
        }
    });
}

int crisb_debug_read(crisb_renderer* r, int id, void* dst, size_t bytes) {
    return guarded([&] {
        require(r && dst, "null argument");
        size_t want = 0;
        if (crisb_debug_size(r, id, &want) != CRISB_OK) throw Error(CRISB_ERR_INVALID_ARGUMENT, g_last_error);
        require(bytes == want, "debug: size mismatch");
        check(cudaDeviceSynchronize(), "sync");
        const size_t P = r->P();
        switch (id) {
            case CRISB_BUF_PREFIX_RES_FRONT:
                check(cudaMemcpy(dst, r->pres[r->front].p, bytes, cudaMemcpyDeviceToHost), "read");
                break;
            case CRISB_BUF_PREFIX_RES_BACK:
                check(cudaMemcpy(dst, r->pres[r->back].p, bytes, cudaMemcpyDeviceToHost), "read");
                break;
            case CRISB_BUF_CANON_PREFIX:
                check(cudaMemcpy(dst, r->canon_prefix.p, bytes, cudaMemcpyDeviceToHost), "read");
                break;
            case CRISB_BUF_SUFFIX_RES_FRONT:
            case CRISB_BUF_SUFFIX_RES_BACK:
                check(cudaMemcpy(dst, r->sres[r->scur].p, bytes, cudaMemcpyDeviceToHost), "read");
                break;
            case CRISB_BUF_CANON_SUFFIX: {
                std::vector<crisb_suffix_res_rec> tmp(P);
                check(cudaMemcpy(tmp.data(), r->canon_suffix.p, P * sizeof(crisb_suffix_res_rec),
                                 cudaMemcpyDeviceToHost),
                      "read");
                auto* o = static_cast<crisb_suffix_rec*>(dst);
                for (size_t i = 0; i < P; ++i) o[i] = tmp[i].sample;
                break;
            }
            case CRISB_BUF_GBUFFER:
                check(cudaMemcpy(dst, r->gbuf.p, bytes, cudaMemcpyDeviceToHost), "read");
                break;
            case CRISB_BUF_NEIGHBORS:
                if (bytes) check(cudaMemcpy(dst, r->neighbors.p, bytes, cudaMemcpyDeviceToHost), "read");
                break;
            case CRISB_BUF_NEIGHBOR_COUNT:
                check(cudaMemcpy(dst, r->neigh_count.p, bytes, cudaMemcpyDeviceToHost), "read");
                break;
            default: break;
        }
    });
}

int crisb_abi_sizes(uint32_t* out, uint32_t n) {
    const uint32_t sizes[] = {
        sizeof(crisb_material),    sizeof(crisb_mesh),         sizeof(crisb_instance),     sizeof(crisb_emitter),
        sizeof(crisb_scene_desc),  sizeof(crisb_camera),       sizeof(crisb_camera_data),  sizeof(crisb_params),
        sizeof(crisb_hit_rec),     sizeof(crisb_prefix_rec),   sizeof(crisb_prefix_res_rec), sizeof(crisb_suffix_rec),
        sizeof(crisb_suffix_res_rec), sizeof(crisb_gbuffer_rec), sizeof(crisb_neighbor_rec), sizeof(crisb_trace_hit),
        sizeof(crisb_stats), sizeof(crisb_hit16_rec), sizeof(crisb_prefix_res16_rec), sizeof(crisb_suffix_res16_rec),
        sizeof(crisb_tuning), sizeof(crisb_bvh_info)};
    const uint32_t count = sizeof(sizes) / sizeof(sizes[0]);
    if (!out) return static_cast<int>(count);
    for (uint32_t i = 0; i < n && i < count; ++i) out[i] = sizes[i];
    return static_cast<int>(count);
}

}  // extern "C"
