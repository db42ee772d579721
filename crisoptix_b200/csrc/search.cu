// search.cu -- the prefix-endpoint neighbour search as a standalone operation:
// build the search structure over caller-given entries, then answer a batch
// of query points.  The renderer runs the same query inside its final gather.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "context.h"
#include "knn.cuh"
#include "radix_sort.h"

namespace crisb {

// passes.cu / api.cu
void launch_lbvh_hierarchy(const lbvh::Work& w, uint32_t cap, int leaf_max, cudaStream_t st);
void set_last_error(const std::string& msg);

namespace search {

constexpr int kBlock = 128;
constexpr int kLeafMax = 8;

inline unsigned grid(uint32_t n) { return (std::max<uint32_t>(n, 1) + kBlock - 1) / kBlock; }

// Scratch of one search over `cap` entries, carved from one block of device
// memory.
struct Scratch {
    lbvh::Work w;
    float4* leaf;
    unsigned int* bounds;
    void* sort_temp;
    size_t sort_bytes;
};

inline size_t align256(size_t v) { return (v + 255) & ~static_cast<size_t>(255); }

// Bytes needed for `cap` entries; with base != nullptr also fills `s`.
inline size_t layout(uint32_t cap, size_t sort_bytes, char* base, Scratch* s) {
    const size_t c = std::max<uint32_t>(cap, 2);
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off = align256(off + bytes);
        return p;
    };
    char* keys_in = take(c * 8);
    char* keys = take(c * 8);
    char* inner_parent = take(c * 4);
    char* leaf_parent = take(c * 4);
    char* inner_left = take(c * 4);
    char* inner_right = take(c * 4);
    char* range_lo = take(c * 4);
    char* range_hi = take(c * 4);
    char* flags = take(c * 4);
    char* inner_box = take(c * sizeof(lbvh::Box));
    char* leaf_box = take(c * sizeof(lbvh::Box));
    char* order = take(c * 4);
    char* nodes = take(c * sizeof(BvhNode));
    char* leaf = take(c * sizeof(float4));
    char* n = take(16);
    char* bounds = take(32);
    char* err = take(16);
    char* temp = take(sort_bytes);
    if (base && s) {
        s->w.keys_in = reinterpret_cast<uint64_t*>(keys_in);
        s->w.keys = reinterpret_cast<uint64_t*>(keys);
        s->w.inner_parent = reinterpret_cast<int*>(inner_parent);
        s->w.leaf_parent = reinterpret_cast<int*>(leaf_parent);
        s->w.inner_left = reinterpret_cast<int*>(inner_left);
        s->w.inner_right = reinterpret_cast<int*>(inner_right);
        s->w.range_lo = reinterpret_cast<int*>(range_lo);
        s->w.range_hi = reinterpret_cast<int*>(range_hi);
        s->w.flags = reinterpret_cast<int*>(flags);
        s->w.inner_box = reinterpret_cast<lbvh::Box*>(inner_box);
        s->w.leaf_box = reinterpret_cast<lbvh::Box*>(leaf_box);
        s->w.order = reinterpret_cast<uint32_t*>(order);
        s->w.nodes = reinterpret_cast<BvhNode*>(nodes);
        s->w.n = reinterpret_cast<uint32_t*>(n);
        s->w.err = reinterpret_cast<int*>(err);
        s->leaf = reinterpret_cast<float4*>(leaf);
        s->bounds = reinterpret_cast<unsigned int*>(bounds);
        s->sort_temp = temp;
        s->sort_bytes = sort_bytes;
    }
    return off;
}

inline size_t sort_temp_bytes(uint32_t cap) { return rsort::temp_bytes(std::max<uint32_t>(cap, 2)); }

__global__ void k_init(unsigned int* ob, uint32_t* n, int* err) {
    if (threadIdx.x < 3) ob[threadIdx.x] = float_to_ordered(INFINITY);
    else if (threadIdx.x < 6) ob[threadIdx.x] = float_to_ordered(-INFINITY);
    if (threadIdx.x == 0) {
        *n = 0;
        *err = 0;
    }
}

// bounds and count of the entries with a radius >= 0
__global__ void k_bounds(const float4* entries, uint32_t n_entries, unsigned int* ob, uint32_t* count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float4 e = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    if (i < n_entries) e = entries[i];
    const bool valid = i < n_entries && e.w >= 0.0f && !nonfinite(V3{e.x, e.y, e.z}) && !isnan(e.w);
    __shared__ float smin[3][kBlock], smax[3][kBlock];
    __shared__ uint32_t scount[kBlock];
    smin[0][threadIdx.x] = valid ? e.x : INFINITY;
    smin[1][threadIdx.x] = valid ? e.y : INFINITY;
    smin[2][threadIdx.x] = valid ? e.z : INFINITY;
    smax[0][threadIdx.x] = valid ? e.x : -INFINITY;
    smax[1][threadIdx.x] = valid ? e.y : -INFINITY;
    smax[2][threadIdx.x] = valid ? e.z : -INFINITY;
    scount[threadIdx.x] = valid ? 1u : 0u;
    __syncthreads();
    for (int off = kBlock / 2; off > 0; off >>= 1) {
        if (threadIdx.x < off) {
            for (int a = 0; a < 3; ++a) {
                smin[a][threadIdx.x] = fminf(smin[a][threadIdx.x], smin[a][threadIdx.x + off]);
                smax[a][threadIdx.x] = fmaxf(smax[a][threadIdx.x], smax[a][threadIdx.x + off]);
            }
            scount[threadIdx.x] += scount[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && scount[0] > 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(&ob[a], float_to_ordered(smin[a][0]));
            atomicMax(&ob[3 + a], float_to_ordered(smax[a][0]));
        }
        atomicAdd(count, scount[0]);
    }
}

__global__ void k_keys(const float4* entries, uint32_t n_entries, const unsigned int* ob, uint64_t* keys) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_entries) return;
    const float4 e = entries[i];
    uint64_t key = ~0ull;
    if (e.w >= 0.0f && !nonfinite(V3{e.x, e.y, e.z}) && !isnan(e.w)) {
        float lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
            lo[a] = ordered_to_float(ob[a]);
            hi[a] = ordered_to_float(ob[3 + a]);
        }
        key = lbvh::morton_key(lo, hi, e.x, e.y, e.z, i);
    }
    keys[i] = key;
}

__global__ void k_leaves(const float4* entries, lbvh::Work w, float4* leaf) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= *w.n) return;
    const uint32_t idx = static_cast<uint32_t>(w.keys[i] & 0xFFFFFFFFull);
    w.order[i] = idx;
    const float4 e = entries[idx];
    leaf[i] = e;
    w.leaf_box[i] = entry_box(e);
}

// Device error word of the standalone searches: the kDevErr* bits of every
// query that stopped early since the word was last read.  Each CUDA context
// that loads the library has its own copy, zero at load.
__device__ int g_search_err;

// visit cap per query; 0 selects kKnnMaxVisits (set only by tests)
std::atomic<uint32_t> g_visit_cap{0};

__global__ void k_query(KnnView v, const float* queries, uint32_t n_queries, uint32_t k, uint32_t max_visits,
                        crisb_neighbor_rec* out, uint32_t* count) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n_queries) return;
    NeighborList nl;
    knn_query(v, &g_search_err, V3{queries[3 * q], queries[3 * q + 1], queries[3 * q + 2]}, k, nl, max_visits);
    for (uint32_t j = 0; j < k; ++j) {
        crisb_neighbor_rec r;
        r.pixel = j < nl.count ? nl.pix[j] : 0u;
        r.dist = j < nl.count ? nl.dist[j] : 0.0f;
        out[static_cast<size_t>(q) * k + j] = r;
    }
    count[q] = nl.count;
}

// Enqueue the whole search on `st` using scratch `s` (capacity >= n_entries).
inline cudaError_t run(const Scratch& s, const float4* entries, uint32_t n_entries, const float* queries,
                       uint32_t n_queries, uint32_t k, crisb_neighbor_rec* out, uint32_t* count, cudaStream_t st) {
    k_init<<<1, 32, 0, st>>>(s.bounds, s.w.n, s.w.err);
    if (n_entries > 0) {
        k_bounds<<<grid(n_entries), kBlock, 0, st>>>(entries, n_entries, s.bounds, s.w.n);
        k_keys<<<grid(n_entries), kBlock, 0, st>>>(entries, n_entries, s.bounds, s.w.keys_in);
        const cudaError_t e = rsort::sort_high32(s.w.keys_in, s.w.keys, s.sort_temp, s.sort_bytes, n_entries, st);
        if (e != cudaSuccess) return e;
        k_leaves<<<grid(n_entries), kBlock, 0, st>>>(entries, s.w, s.leaf);
    }
    launch_lbvh_hierarchy(s.w, std::max<uint32_t>(n_entries, 1), kLeafMax, st);
    if (n_queries > 0) {
        const KnnView v{s.w.nodes, s.leaf, s.w.order, s.w.n};
        const uint32_t cap = g_visit_cap.load(std::memory_order_relaxed);
        k_query<<<grid(n_queries), kBlock, 0, st>>>(v, queries, n_queries, k, cap ? cap : kKnnMaxVisits, out,
                                                    count);
    }
    return cudaGetLastError();
}

inline int fail(int code, const std::string& msg) {
    set_last_error(msg);
    return code;
}

inline int validate(const float* entries, uint32_t n_entries, const float* queries, uint32_t n_queries, uint32_t k,
                    const crisb_neighbor_rec* out, const uint32_t* count) {
    if ((n_entries > 0 && !entries) || (n_queries > 0 && (!queries || !out || !count)))
        return fail(CRISB_ERR_INVALID_ARGUMENT, "endpoint search: null array");
    if (k < 1 || k > CRISB_MAX_GATHER_M - 1) return fail(CRISB_ERR_INVALID_ARGUMENT, "endpoint search: k must be in [1, 31]");
    if (n_entries >= (1u << 31)) return fail(CRISB_ERR_INVALID_ARGUMENT, "endpoint search: too many entries");
    if (reinterpret_cast<uintptr_t>(entries) % 16 != 0)
        return fail(CRISB_ERR_INVALID_ARGUMENT, "endpoint search: entries must be 16-byte aligned");
    if (reinterpret_cast<uintptr_t>(out) % alignof(crisb_neighbor_rec) != 0 ||
        reinterpret_cast<uintptr_t>(count) % alignof(uint32_t) != 0 ||
        reinterpret_cast<uintptr_t>(queries) % alignof(float) != 0)
        return fail(CRISB_ERR_INVALID_ARGUMENT, "endpoint search: misaligned queries, out or count array");
    return CRISB_OK;
}

}  // namespace search
}  // namespace crisb

using namespace crisb;

extern "C" int crisb_endpoint_search(const float* entries_dev, uint32_t n_entries, const float* queries_dev,
                                     uint32_t n_queries, uint32_t k, crisb_neighbor_rec* out_dev, uint32_t* count_dev,
                                     void* stream) {
    int rc = search::validate(entries_dev, n_entries, queries_dev, n_queries, k, out_dev, count_dev);
    if (rc != CRISB_OK) return rc;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t sort_bytes = search::sort_temp_bytes(n_entries);
    const size_t bytes = search::layout(n_entries, sort_bytes, nullptr, nullptr);
    void* base = nullptr;
    cudaError_t e = cudaMallocAsync(&base, bytes, st);
    if (e != cudaSuccess)
        return search::fail(e == cudaErrorMemoryAllocation ? CRISB_ERR_OUT_OF_MEMORY : CRISB_ERR_CUDA,
                            std::string("endpoint search: cudaMallocAsync: ") + cudaGetErrorString(e));
    search::Scratch s;
    search::layout(n_entries, sort_bytes, static_cast<char*>(base), &s);
    e = search::run(s, reinterpret_cast<const float4*>(entries_dev), n_entries, queries_dev, n_queries, k, out_dev,
                    count_dev, st);
    const cudaError_t e2 = cudaFreeAsync(base, st);
    if (e != cudaSuccess || e2 != cudaSuccess)
        return search::fail(CRISB_ERR_CUDA, std::string("endpoint search: ") +
                                                cudaGetErrorString(e != cudaSuccess ? e : e2));
    return CRISB_OK;
}

// ---- allocation-free variant -------------------------------------------------------
// Scratch for crisb_endpoint_search_noalloc: one static device array that
// every GPU loading this library holds until the process exits.  Host code
// only sees a stand-in symbol for it; its device address comes from
// cudaGetSymbolAddress, looked up once per CUDA context (an address is only
// valid in the context it was looked up in).
namespace {

constexpr size_t kNoAllocScratchBytes = 8u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
std::vector<std::pair<unsigned long long, void*>> g_noalloc_base;  // (context id, address)

// device address of the scratch array in the current context (the first call
// in a context does the lookup and checks that the largest accepted search
// fits)
int noalloc_scratch(void** out) {
    unsigned long long ctx = 0;
    cudaError_t e = current_context_id(&ctx);
    if (e != cudaSuccess)
        return search::fail(CRISB_ERR_CUDA, std::string("endpoint search (no-alloc): no current context: ") +
                                                cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    for (const auto& b : g_noalloc_base)
        if (b.first == ctx) {
            *out = b.second;
            return CRISB_OK;
        }
    const size_t need = search::layout(CRISB_NOALLOC_MAX_ENTRIES, search::sort_temp_bytes(CRISB_NOALLOC_MAX_ENTRIES),
                                       nullptr, nullptr);
    if (need > kNoAllocScratchBytes)
        return search::fail(CRISB_ERR_NOT_SUPPORTED, "endpoint search (no-alloc): scratch array too small");
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return search::fail(CRISB_ERR_CUDA,
                            std::string("endpoint search (no-alloc): cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_noalloc_base.emplace_back(ctx, p);
    *out = p;
    return CRISB_OK;
}

}  // namespace

extern "C" int crisb_endpoint_search_noalloc(const float* entries_dev, uint32_t n_entries, const float* queries_dev,
                                             uint32_t n_queries, uint32_t k, crisb_neighbor_rec* out_dev,
                                             uint32_t* count_dev, void* stream) {
    int rc = search::validate(entries_dev, n_entries, queries_dev, n_queries, k, out_dev, count_dev);
    if (rc != CRISB_OK) return rc;
    if (n_entries > CRISB_NOALLOC_MAX_ENTRIES)
        return search::fail(CRISB_ERR_INVALID_ARGUMENT,
                            "endpoint search (no-alloc): n_entries " + std::to_string(n_entries) +
                                " exceeds the maximum " + std::to_string(CRISB_NOALLOC_MAX_ENTRIES));
    void* base = nullptr;
    rc = noalloc_scratch(&base);
    if (rc != CRISB_OK) return rc;
    const size_t sort_bytes = search::sort_temp_bytes(n_entries);
    if (search::layout(n_entries, sort_bytes, nullptr, nullptr) > kNoAllocScratchBytes)
        return search::fail(CRISB_ERR_NOT_SUPPORTED, "endpoint search (no-alloc): scratch does not fit");
    search::Scratch s;
    search::layout(n_entries, sort_bytes, static_cast<char*>(base), &s);
    const cudaError_t e = search::run(s, reinterpret_cast<const float4*>(entries_dev), n_entries, queries_dev,
                                      n_queries, k, out_dev, count_dev, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess)
        return search::fail(CRISB_ERR_CUDA, std::string("endpoint search (no-alloc): ") + cudaGetErrorString(e));
    return CRISB_OK;
}

extern "C" int crisb_endpoint_search_status(void* stream) {
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    int word = 0;
    static const int zero = 0;
    cudaError_t e = cudaMemcpyFromSymbolAsync(&word, search::g_search_err, sizeof word, 0, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyToSymbolAsync(search::g_search_err, &zero, sizeof zero, 0,
                                                      cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess)
        return search::fail(CRISB_ERR_CUDA, std::string("endpoint search status: ") + cudaGetErrorString(e));
    if (word != 0)
        return search::fail(CRISB_ERR_DEVICE_FAULT,
                            std::string("endpoint search: a query stopped early (") +
                                ((word & kDevErrKnn) ? "visit cap" : "") +
                                ((word & kDevErrKnn) && (word & kDevErrStack) ? ", " : "") +
                                ((word & kDevErrStack) ? "stack depth" : "") + "); its neighbour list is incomplete");
    return CRISB_OK;
}

extern "C" int crisb_endpoint_search_set_visit_cap(uint32_t max_visits) {
    search::g_visit_cap.store(max_visits, std::memory_order_relaxed);
    return CRISB_OK;
}
