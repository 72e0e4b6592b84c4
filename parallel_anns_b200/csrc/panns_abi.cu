// C ABI of panns_b200 (declared in include/panns_b200.h): loaders, the HBM
// layout of the base vectors and the graph, init-id generation, the batched
// search launch and recall. Host code is C++; the hot path is search_kernel.cuh.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/panns_b200.h"
#include "../../include/panns_learned.h"
#include "graph_types.h"
#include "learned.h"
#include "search_kernel.cuh"
#include "block_kernel.cuh"
#include "gt_kernel.cuh"
#include "pss_kernel.cuh"
#include "kernels.h"

using namespace panns;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define CU(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(PANNS_ECUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
    } while (0)

// Chain-major padding: the reference's lane accumulator c visits the terms
// c, c+8, c+16, ... (after the last 8 elements when d % 16 == 8). Term k of
// chain c is stored at float (8 * (k / 4) + c) * 4 + k % 4 of the padded row.
__host__ __device__ inline int chain_term_element(int d, int c, int k) {
    const int DR = d % 16, DD = d - DR;
    const int nterms = d / 8;
    if (k >= nterms) return -1;
    if (DR) return k == 0 ? DD + c : c + 8 * (k - 1);
    return c + 8 * k;
}

// out row r = chain-major copy of raw row (rowmap ? rowmap[r] : r).
__global__ void permute_rows_kernel(const float *__restrict__ raw, float *__restrict__ out,
                                    uint64_t rows, int d, int dpad,
                                    const uint32_t *__restrict__ rowmap) {
    const uint64_t total = rows * (uint64_t) dpad;
    for (uint64_t t = blockIdx.x * (uint64_t) blockDim.x + threadIdx.x; t < total;
         t += (uint64_t) gridDim.x * blockDim.x) {
        const uint64_t r = t / dpad;
        const uint64_t src = rowmap ? rowmap[r] : r;
        const int p = (int) (t % dpad);
        const int chunk = p >> 2, i = chunk >> 3, c = chunk & 7;
        const int k = 4 * i + (p & 3);
        const int e = chain_term_element(d, c, k);
        out[t] = e >= 0 ? raw[src * d + e] : 0.0f;
    }
}


// ||v||^2 from the chain-major rows: lane c = FMA chain over its terms, then
// the lanes summed 0..7 (core/Searching.202102022027.PSS_v5.dist_thresh.profiling.cpp:294-335).
__global__ void norms_kernel(const float *__restrict__ vec, float *__restrict__ norms, uint32_t n,
                             int dpad) {
    const int CL = dpad / 32;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float *row = vec + (size_t) v * dpad;
        float acc[8];
        for (int c = 0; c < 8; ++c) {
            float a = 0.0f;
            for (int i = 0; i < CL; ++i)
                for (int j = 0; j < 4; ++j) {
                    const float x = row[(8 * i + c) * 4 + j];
                    a = __fmaf_rn(x, x, a);
                }
            acc[c] = a;
        }
        float s = acc[0];
        for (int c = 1; c < 8; ++c) s = __fadd_rn(s, acc[c]);
        norms[v] = s;
    }
}

// Per-dimension absolute maximum (FP8 scales), as float bits (non-negative
// floats order like their bit patterns).
__global__ void absmax_kernel(const float *__restrict__ raw, uint64_t n, int d, unsigned int *amax) {
    const uint64_t total = n * (uint64_t) d;
    for (uint64_t t = blockIdx.x * (uint64_t) blockDim.x + threadIdx.x; t < total;
         t += (uint64_t) gridDim.x * blockDim.x)
        atomicMax(amax + (t % d), __float_as_uint(fabsf(raw[t])));
}

// Reduced copy, natural element order, row u = original row rowmap[u], padded
// to dpad with zeros: BF16 (round to nearest even) or FP8 E4M3 of x / scale
// (saturating). Then ||v^||^2 of the dequantised row.
__global__ void quantize_rows_kernel(const float *__restrict__ raw, void *out, float *norms_lo,
                                     uint32_t n, int d, int dpad, const uint32_t *__restrict__ rowmap,
                                     int store, const float *__restrict__ scales) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        const float *x = raw + (uint64_t) rowmap[u] * d;
        float s = 0.f;
        for (int e = 0; e < dpad; ++e) {
            const float v = e < d ? x[e] : 0.f;
            float back;
            if (store == PANNS_STORE_BF16) {
                const __nv_bfloat16 b = __float2bfloat16_rn(v);
                reinterpret_cast<__nv_bfloat16 *>(out)[(uint64_t) u * dpad + e] = b;
                back = __bfloat162float(b);
            } else {
                const __nv_fp8_storage_t f = __nv_cvt_float_to_fp8(v / scales[e], __NV_SATFINITE, __NV_E4M3);
                reinterpret_cast<__nv_fp8_storage_t *>(out)[(uint64_t) u * dpad + e] = f;
                const __half_raw hr = __nv_cvt_fp8_to_halfraw(f, __NV_E4M3);
                back = __half2float(*reinterpret_cast<const __half *>(&hr)) * scales[e];
            }
            s = fmaf(back, back, s);
        }
        norms_lo[u] = s;
    }
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t n = 0;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    cudaError_t ensure(size_t count) {
        if (count <= n && p) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) n = count;
        else p = nullptr;
        return e;
    }
};

}  // namespace

int panns::set_error(int code, const std::string &msg) { return fail(code, msg); }

struct panns_index {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // base vectors (raw rows stay on the device until the index is finalised)
    uint32_t n = 0, d = 0, dpad = 0, storage = 0;
    DevBuf<float> base_raw, vec, norms;
    DevBuf<uint8_t> vec_lo;         // reduced copy (BF16 or FP8 rows)
    DevBuf<float> norms_lo, scales; // its norms; FP8 per-dimension scales
    bool ready = false;             // vec/norms/head built for the current base + graph
    std::vector<uint32_t> perm, inv;  // device id -> original id, and back
    DevBuf<uint32_t> orig;
    // graph
    uint32_t width = 0, entry = 0, gn = 0, max_deg = 0;
    std::vector<uint64_t> off;
    std::vector<uint32_t> nbrs;
    DevBuf<uint32_t> head, ovf;
    DevBuf<uint64_t> ovf_off;
    // queries
    uint32_t nq = 0, qd = 0;
    DevBuf<float> queries;  // chain-major
    DevBuf<float> hq;       // chain-major staging of host-pointer queries
    // scratch
    DevBuf<float> raw;      // staging for permutation
    DevBuf<uint32_t> visited, dirty, counter, error, init, out;
    DevBuf<uint4> stats;
    uint32_t vis_slots = 0, vis_words = 0, dirty_cap = 0;
    std::vector<uint4> h_stats;
    DevBuf<uint32_t> lq;        // per-query queue lengths of the current call
    DevBuf<uint32_t> init_def;  // default PANNS init list (device ids) for init_def_L
    uint32_t init_def_L = 0;
    DevBuf<float> dq;           // chain-major copy of device-pointer queries
    // Captured launch (PANNS_FLAG_CUDA_GRAPH): replayed while its key matches.
    cudaGraphExec_t gexec = nullptr;
    std::vector<uint8_t> gkey;
    // Learned entry / L-budget network (PANNS_FLAG_LEARNED).
    bool has_mlp = false;
    MlpDev mlp{};                  // the network (device pointers) and decision rule
    DevBuf<uint16_t> mlp_w;        // BF16 weights, inference layout
    DevBuf<float> mlp_f;           // biases and regressor
    DevBuf<uint32_t> mlp_rep;      // representatives (device ids)
    DevBuf<float> mlp_scratch;     // batched inference: X, H1, H2, Z of one chunk of queries
    uint32_t mlp_chunk = 0;        // queries per chunk the scratch holds
    DevBuf<uint32_t> mlp_record;   // per-query decisions of the last call
    uint32_t mlp_rec_cap = 0, mlp_last_nq = 0;
};

extern "C" {

const char *panns_last_error(void) { return g_err.c_str(); }
uint32_t panns_version(void) { return (1u << 16) | 0u; }

int panns_open(panns_index **out, int device) {
    if (!out) return fail(PANNS_EINVAL, "panns_open: out is NULL");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(PANNS_ECUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= count) return fail(PANNS_EINVAL, "panns_open: bad device index");
    CU(cudaSetDevice(device));
    cudaDeviceProp prop;
    CU(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return fail(PANNS_ECUDA, "panns_b200 is built for sm_100a (B200); found sm_" +
                                     std::to_string(prop.major) + std::to_string(prop.minor));
    std::unique_ptr<panns_index> h(new panns_index());
    h->device = device;
    h->num_sms = prop.multiProcessorCount;
    CU(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    CU(cudaEventCreate(&h->ev0));
    CU(cudaEventCreate(&h->ev1));
    *out = h.release();
    return PANNS_OK;
}

int panns_close(panns_index *h) {
    if (!h) return PANNS_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return PANNS_OK;
}

static int upload_chain_major(panns_index *h, const float *rows, uint64_t count, uint32_t d,
                              DevBuf<float> &dst) {
    const uint32_t dpad = 32u * chain_blocks(d);
    CU(h->raw.ensure(count * d));
    CU(dst.ensure(count * dpad));
    CU(cudaMemcpyAsync(h->raw.p, rows, count * d * sizeof(float), cudaMemcpyHostToDevice, h->stream));
    const uint64_t total = count * dpad;
    const int blocks = (int) std::min<uint64_t>((total + 255) / 256, (uint64_t) h->num_sms * 32);
    permute_rows_kernel<<<std::max(blocks, 1), 256, 0, h->stream>>>(h->raw.p, dst.p, count, (int) d,
                                                                   (int) dpad, nullptr);
    CU(cudaGetLastError());
    return PANNS_OK;
}

int panns_set_base(panns_index *h, const float *data, uint32_t n, uint32_t d, uint32_t storage) {
    if (!h || !data) return fail(PANNS_EINVAL, "panns_set_base: NULL argument");
    if (n == 0 || d == 0) return fail(PANNS_EINVAL, "panns_set_base: empty base");
    if (d % 8) return fail(PANNS_EINVAL, "panns_set_base: d must be a multiple of 8");
    if (d > 256) return fail(PANNS_EINVAL, "panns_set_base: d > 256 is not supported");
    if (n > 0x7fffffffu) return fail(PANNS_EINVAL, "panns_set_base: n must be < 2^31");
    if (storage > PANNS_STORE_FP8) return fail(PANNS_EINVAL, "panns_set_base: unknown storage");
    if (h->qd && h->qd != d) return fail(PANNS_EINVAL, "panns_set_base: dimension differs from the queries");
    if (h->gn && h->gn != n)
        return fail(PANNS_EINVAL, "panns_set_base: base has " + std::to_string(n) +
                                      " vectors, the graph has " + std::to_string(h->gn) + " vertices");
    CU(cudaSetDevice(h->device));
    CU(h->base_raw.ensure((size_t) n * d));
    CU(cudaMemcpyAsync(h->base_raw.p, data, (size_t) n * d * sizeof(float), cudaMemcpyHostToDevice,
                       h->stream));
    CU(cudaStreamSynchronize(h->stream));
    h->n = n;
    h->d = d;
    h->dpad = 32u * chain_blocks(d);
    h->storage = storage;
    h->ready = false;
    return PANNS_OK;
}

static int read_fvecs(const char *path, std::vector<float> &v, uint32_t &n, uint32_t &d) {
    FILE *f = fopen(path, "rb");
    if (!f) return fail(PANNS_EIO, std::string("cannot open ") + path);
    uint32_t dim = 0;
    if (fread(&dim, 4, 1, f) != 1) {
        fclose(f);
        return fail(PANNS_EIO, std::string("empty fvecs file ") + path);
    }
    fseek(f, 0, SEEK_END);
    const uint64_t sz = (uint64_t) ftell(f);
    fseek(f, 0, SEEK_SET);
    if (dim == 0 || sz % (4ull * (dim + 1))) {
        fclose(f);
        return fail(PANNS_EIO, std::string("fvecs size is not a whole number of rows: ") + path);
    }
    const uint64_t rows = sz / (4ull * (dim + 1));
    if (rows > 0x7fffffffull) {
        fclose(f);
        return fail(PANNS_EIO, "fvecs: too many rows");
    }
    v.resize(rows * dim);
    std::vector<uint32_t> rec(dim + 1);
    for (uint64_t i = 0; i < rows; ++i) {
        if (fread(rec.data(), 4, dim + 1, f) != dim + 1 || rec[0] != dim) {
            fclose(f);
            return fail(PANNS_EIO, std::string("fvecs row ") + std::to_string(i) + " is malformed");
        }
        memcpy(v.data() + i * dim, rec.data() + 1, 4ull * dim);
    }
    fclose(f);
    n = (uint32_t) rows;
    d = dim;
    return PANNS_OK;
}

int panns_load_fvecs_base(panns_index *h, const char *path, uint32_t storage) {
    if (!h || !path) return fail(PANNS_EINVAL, "panns_load_fvecs_base: NULL argument");
    std::vector<float> v;
    uint32_t n = 0, d = 0;
    int rc = read_fvecs(path, v, n, d);
    if (rc) return rc;
    return panns_set_base(h, v.data(), n, d, storage);
}

int panns_set_queries(panns_index *h, const float *queries, uint32_t nq, uint32_t d) {
    if (!h || (!queries && nq)) return fail(PANNS_EINVAL, "panns_set_queries: NULL argument");
    if (d % 8 || d == 0 || d > 256) return fail(PANNS_EINVAL, "panns_set_queries: bad dimension");
    if (h->d && d != h->d) return fail(PANNS_EINVAL, "panns_set_queries: dimension differs from the base");
    CU(cudaSetDevice(h->device));
    if (nq) {
        int rc = upload_chain_major(h, queries, nq, d, h->queries);
        if (rc) return rc;
        CU(cudaStreamSynchronize(h->stream));
        h->raw.release();
    }
    h->nq = nq;
    h->qd = d;
    return PANNS_OK;
}

int panns_load_fvecs_queries(panns_index *h, const char *path) {
    if (!h || !path) return fail(PANNS_EINVAL, "panns_load_fvecs_queries: NULL argument");
    std::vector<float> v;
    uint32_t n = 0, d = 0;
    int rc = read_fvecs(path, v, n, d);
    if (rc) return rc;
    return panns_set_queries(h, v.data(), n, d);
}

int panns_set_graph(panns_index *h, uint32_t width, uint32_t entry, const uint64_t *offsets,
                    const uint32_t *nbrs, uint32_t n) {
    if (!h || !offsets || (!nbrs && offsets[n])) return fail(PANNS_EINVAL, "panns_set_graph: NULL argument");
    if (n == 0) return fail(PANNS_EINVAL, "panns_set_graph: empty graph");
    if (h->n && n != h->n)
        return fail(PANNS_EINVAL, "panns_set_graph: graph has " + std::to_string(n) +
                                      " vertices, the base has " + std::to_string(h->n));
    if (entry >= n) return fail(PANNS_EINVAL, "panns_set_graph: entry vertex out of range");
    if (offsets[0] != 0) return fail(PANNS_EINVAL, "panns_set_graph: offsets[0] must be 0");
    for (uint32_t v = 0; v < n; ++v)
        if (offsets[v + 1] < offsets[v]) return fail(PANNS_EINVAL, "panns_set_graph: offsets not monotone");
    const uint64_t E = offsets[n];
    for (uint64_t e = 0; e < E; ++e)
        if (nbrs[e] >= n)
            return fail(PANNS_EINVAL, "panns_set_graph: neighbour id " + std::to_string(nbrs[e]) +
                                          " >= N");
    h->off.assign(offsets, offsets + n + 1);
    h->nbrs.assign(nbrs, nbrs + E);
    h->max_deg = 0;
    for (uint32_t v = 0; v < n; ++v) h->max_deg = std::max<uint32_t>(h->max_deg, (uint32_t) (offsets[v + 1] - offsets[v]));
    h->width = width;
    h->entry = entry;
    h->gn = n;
    h->ready = false;
    return PANNS_OK;
}

// Build the search layout from the current base + graph: the locality order
// (vertices grouped by their nearest of C pivot vertices, original id order
// inside a group), chain-major rows and norms in that order, head rows and
// overflow lists in device ids.
static int finalize(panns_index *h) {
    if (h->ready) return PANNS_OK;
    if (!h->n || !h->base_raw.p) return fail(PANNS_ESTATE, "search: no base vectors loaded");
    if (!h->gn) return fail(PANNS_ESTATE, "search: no graph loaded");
    if (h->gn != h->n) return fail(PANNS_ESTATE, "search: graph and base sizes differ");
    const uint32_t n = h->n;
    CU(cudaSetDevice(h->device));
    h->perm.resize(n);
    h->inv.resize(n);
    const char *ord = getenv("PANNS_LAYOUT_ORDER");
    const bool identity = (ord && std::string(ord) == "identity") || n < 4096;
    if (identity) {
        for (uint32_t v = 0; v < n; ++v) h->perm[v] = h->inv[v] = v;
    } else {
        const uint32_t C = std::max(1u, std::min(4096u, n / 256));
        std::vector<uint32_t> piv(C), cell(n);
        for (uint32_t p = 0; p < C; ++p) piv[p] = (uint32_t) (((uint64_t) p * n) / C);
        DevBuf<uint32_t> dpiv, dcell;
        CU(dpiv.ensure(C));
        CU(dcell.ensure(n));
        CU(cudaMemcpyAsync(dpiv.p, piv.data(), C * 4ull, cudaMemcpyHostToDevice, h->stream));
        int rc = panns::nearest_center(h->base_raw.p, n, h->d, dpiv.p, C, dcell.p, h->stream);
        if (rc) return rc;
        CU(cudaMemcpyAsync(cell.data(), dcell.p, n * 4ull, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
        std::vector<uint32_t> start(C + 1, 0);
        for (uint32_t v = 0; v < n; ++v) start[cell[v] + 1]++;
        for (uint32_t c = 0; c < C; ++c) start[c + 1] += start[c];
        for (uint32_t v = 0; v < n; ++v) h->perm[start[cell[v]]++] = v;
        for (uint32_t u = 0; u < n; ++u) h->inv[h->perm[u]] = u;
    }
    CU(h->orig.ensure(n));
    CU(cudaMemcpyAsync(h->orig.p, h->perm.data(), n * 4ull, cudaMemcpyHostToDevice, h->stream));
    // rows and norms
    CU(h->vec.ensure((size_t) n * h->dpad));
    {
        const uint64_t total = (uint64_t) n * h->dpad;
        const int blocks = (int) std::min<uint64_t>((total + 255) / 256, (uint64_t) h->num_sms * 32);
        permute_rows_kernel<<<std::max(blocks, 1), 256, 0, h->stream>>>(h->base_raw.p, h->vec.p, n,
                                                                       (int) h->d, (int) h->dpad,
                                                                       h->orig.p);
        CU(cudaGetLastError());
    }
    CU(h->norms.ensure(n));
    {
        const int blocks = std::max(1, (int) std::min<uint32_t>((n + 255) / 256, h->num_sms * 32u));
        norms_kernel<<<blocks, 256, 0, h->stream>>>(h->vec.p, h->norms.p, n, (int) h->dpad);
        CU(cudaGetLastError());
    }
    if (h->storage != PANNS_STORE_FP32) {
        const size_t esz = h->storage == PANNS_STORE_BF16 ? 2 : 1;
        CU(h->vec_lo.ensure((size_t) n * h->dpad * esz));
        CU(h->norms_lo.ensure(n));
        CU(h->scales.ensure(h->dpad));
        std::vector<float> sc(h->dpad, 1.0f);
        if (h->storage == PANNS_STORE_FP8) {
            DevBuf<unsigned int> amax;
            CU(amax.ensure(h->d));
            CU(cudaMemsetAsync(amax.p, 0, h->d * 4ull, h->stream));
            absmax_kernel<<<h->num_sms * 8, 256, 0, h->stream>>>(h->base_raw.p, n, (int) h->d, amax.p);
            CU(cudaGetLastError());
            std::vector<unsigned int> am(h->d);
            CU(cudaMemcpyAsync(am.data(), amax.p, h->d * 4ull, cudaMemcpyDeviceToHost, h->stream));
            CU(cudaStreamSynchronize(h->stream));
            for (uint32_t e = 0; e < h->d; ++e) {
                float m;
                memcpy(&m, &am[e], 4);
                sc[e] = m > 0.f ? m / 448.0f : 1.0f;  // E4M3 largest finite value: 448
            }
        }
        CU(cudaMemcpyAsync(h->scales.p, sc.data(), h->dpad * 4ull, cudaMemcpyHostToDevice, h->stream));
        const int blocks = std::max(1, (int) std::min<uint32_t>((n + 127) / 128, h->num_sms * 16u));
        quantize_rows_kernel<<<blocks, 128, 0, h->stream>>>(h->base_raw.p, h->vec_lo.p, h->norms_lo.p, n,
                                                            (int) h->d, (int) h->dpad, h->orig.p,
                                                            (int) h->storage, h->scales.p);
        CU(cudaGetLastError());
    }
    // head rows + overflow in device ids
    std::vector<uint32_t> head((size_t) n * kHeadWords, 0u);
    std::vector<uint64_t> ovf_off(n, 0);
    std::vector<uint32_t> ovf;
    for (uint32_t u = 0; u < n; ++u) {
        const uint32_t v = h->perm[u];
        const uint64_t b = h->off[v], deg = h->off[v + 1] - b;
        uint32_t *row = head.data() + (size_t) u * kHeadWords;
        row[0] = (uint32_t) deg;
        const uint64_t h1 = std::min<uint64_t>(deg, kHeadNbrs);
        for (uint64_t s2 = 0; s2 < h1; ++s2) row[1 + s2] = h->inv[h->nbrs[b + s2]];
        if (deg > (uint64_t) kHeadNbrs) {
            ovf_off[u] = ovf.size();
            for (uint64_t s2 = kHeadNbrs; s2 < deg; ++s2) ovf.push_back(h->inv[h->nbrs[b + s2]]);
        }
    }
    CU(h->head.ensure(head.size()));
    CU(h->ovf_off.ensure(n));
    CU(h->ovf.ensure(std::max<size_t>(ovf.size(), 1)));
    CU(cudaMemcpyAsync(h->head.p, head.data(), head.size() * 4, cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(h->ovf_off.p, ovf_off.data(), n * 8ull, cudaMemcpyHostToDevice, h->stream));
    if (!ovf.empty())
        CU(cudaMemcpyAsync(h->ovf.p, ovf.data(), ovf.size() * 4, cudaMemcpyHostToDevice, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    h->init_def_L = 0;
    h->ready = true;
    return PANNS_OK;
}

int panns_load_nsg(panns_index *h, const char *path) {
    if (!h || !path) return fail(PANNS_EINVAL, "panns_load_nsg: NULL argument");
    FILE *f = fopen(path, "rb");
    if (!f) return fail(PANNS_EIO, std::string("cannot open ") + path);
    uint32_t hdr[2];
    if (fread(hdr, 4, 2, f) != 2) {
        fclose(f);
        return fail(PANNS_EIO, std::string("truncated .nsg header: ") + path);
    }
    std::vector<uint64_t> off(1, 0);
    std::vector<uint32_t> nb;
    for (;;) {
        uint32_t deg;
        if (fread(&deg, 4, 1, f) != 1) break;
        const size_t at = nb.size();
        nb.resize(at + deg);
        if (deg && fread(nb.data() + at, 4, deg, f) != deg) {
            fclose(f);
            return fail(PANNS_EIO, std::string("truncated .nsg row ") + std::to_string(off.size() - 1) +
                                       ": " + path);
        }
        off.push_back(nb.size());
    }
    fclose(f);
    const uint32_t n = (uint32_t) (off.size() - 1);
    if (n == 0) return fail(PANNS_EIO, std::string(".nsg has no vertices: ") + path);
    return panns_set_graph(h, hdr[0], hdr[1], off.data(), nb.data(), n);
}

int panns_info(const panns_index *h, uint32_t *n, uint32_t *d, uint32_t *nq, uint32_t *width,
               uint32_t *entry) {
    if (!h) return fail(PANNS_EINVAL, "panns_info: NULL handle");
    if (n) *n = h->n ? h->n : h->gn;
    if (d) *d = h->d;
    if (nq) *nq = h->nq;
    if (width) *width = h->width;
    if (entry) *entry = h->entry;
    return PANNS_OK;
}

}  // extern "C"

// The PANNS init list (prepare_init_ids, PSS.cpp:238-291): the entry's
// neighbours in row order, each once, then entry + 1, entry + 2, ... (wrapping
// at N), skipping the ones already taken. Only entry neighbours can repeat, so
// a scan of the first part replaces a visited array: no allocation, which the
// allocation-free search relies on.
static void fill_init_ids(const panns_index *h, uint32_t L, uint32_t *out) {
    const uint32_t n = h->gn;
    uint32_t end = 0;
    for (uint64_t e = h->off[h->entry]; e < h->off[h->entry + 1] && end < L; ++e) {
        const uint32_t v = h->nbrs[e];
        bool dup = false;
        for (uint32_t i = 0; i < end && !dup; ++i) dup = out[i] == v;
        if (!dup) out[end++] = v;
    }
    const uint32_t from_nbrs = end;
    for (uint32_t t = h->entry + 1; end < L; ++t) {
        if (t == n) t = 0;
        bool dup = false;
        for (uint32_t i = 0; i < from_nbrs && !dup; ++i) dup = out[i] == t;
        if (!dup) out[end++] = t;
    }
}

extern "C" {

int panns_prepare_init_ids(const panns_index *h, uint32_t L, uint32_t *out) {
    if (!h || !out) return fail(PANNS_EINVAL, "panns_prepare_init_ids: NULL argument");
    if (!h->gn) return fail(PANNS_ESTATE, "panns_prepare_init_ids: no graph loaded");
    if (L == 0 || L > h->gn) return fail(PANNS_EINVAL, "panns_prepare_init_ids: need 0 < L <= N");
    fill_init_ids(h, L, out);
    return PANNS_OK;
}

// glibc rand(): the additive feedback generator r[i] = r[i-3] + r[i-31]
// (mod 2^32) over a 31-word table seeded with the Park-Miller sequence
// 16807 * r mod (2^31 - 1) from `seed`, first 310 outputs discarded, each
// output (r >> 1). State layout: table[31], front index, rear index.
static int32_t rand_next(int32_t *st) {
    int32_t *tbl = st;
    int32_t &fi = st[31], &ri = st[32];
    const uint32_t val = (uint32_t) tbl[fi] + (uint32_t) tbl[ri];
    tbl[fi] = (int32_t) val;
    if (++fi >= 31) {
        fi = 0;
        ++ri;
    } else if (++ri >= 31) {
        ri = 0;
    }
    return (int32_t) (val >> 1);
}

int panns_rand_seed(int32_t *st, uint32_t seed) {
    if (!st) return fail(PANNS_EINVAL, "panns_rand_seed: NULL state");
    if (seed == 0) seed = 1;
    st[0] = (int32_t) seed;
    for (int i = 1; i < 31; ++i) {
        const int64_t hi = st[i - 1] / 127773, lo = st[i - 1] % 127773;
        int64_t w = 16807 * lo - 2836 * hi;
        if (w < 0) w += 2147483647;
        st[i] = (int32_t) w;
    }
    st[31] = 3;
    st[32] = 0;
    for (int i = 0; i < 310; ++i) rand_next(st);
    return PANNS_OK;
}

int panns_efanna_init_ids(const panns_index *h, uint32_t L, uint32_t nq, int32_t *st, uint32_t *out) {
    if (!h || !out || !st) return fail(PANNS_EINVAL, "panns_efanna_init_ids: NULL argument");
    if (!h->gn) return fail(PANNS_ESTATE, "panns_efanna_init_ids: no graph loaded");
    const uint32_t n = h->gn;
    if (L == 0 || L > n) return fail(PANNS_EINVAL, "panns_efanna_init_ids: need 0 < L <= N");
    std::vector<uint8_t> flags(n, 0);
    const uint64_t e0 = h->off[h->entry], deg = h->off[h->entry + 1] - e0;
    for (uint32_t q = 0; q < nq; ++q) {
        uint32_t *ids = out + (size_t) q * L;
        uint32_t t = 0;
        for (; t < L && t < deg; ++t) {
            ids[t] = h->nbrs[e0 + t];
            flags[ids[t]] = 1;
        }
        while (t < L) {
            const uint32_t id = (uint32_t) rand_next(st) % n;
            if (flags[id]) continue;
            flags[id] = 1;
            ids[t++] = id;
        }
        for (uint32_t i = 0; i < L; ++i) flags[ids[i]] = 0;
    }
    return PANNS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Search launch
// ---------------------------------------------------------------------------
namespace {

int check_params(panns_index *h, const panns_search_params *p) {
    if (!p) return fail(PANNS_EINVAL, "search: NULL params");
    int rc = finalize(h);
    if (rc) return rc;
    if (p->mode > PANNS_MODE_EFANNA) return fail(PANNS_EINVAL, "search: unknown mode");
    if (p->distance > PANNS_DIST_L2) return fail(PANNS_EINVAL, "search: unknown distance");
    if (p->L == 0 || p->L > h->n) return fail(PANNS_EINVAL, "search: need 0 < L <= N");
    if (p->K == 0 || p->K > p->L) return fail(PANNS_EINVAL, "search: need 0 < K <= L");
    if (p->L > 8192) return fail(PANNS_EINVAL, "search: L > 8192 is not supported");
    if (p->mode == PANNS_MODE_TOP_M && (p->M == 0 || p->M > (uint32_t) kMaxM))
        return fail(PANNS_EINVAL, "search: TOP_M needs 1 <= M <= 64");
    if (p->mode == PANNS_MODE_PSS_V5) {
        if (p->T == 0 || p->X == 0) return fail(PANNS_EINVAL, "search: PSS_V5 needs T >= 1 and X >= 1");
        if (p->T > 64) return fail(PANNS_EINVAL, "search: PSS_V5 needs T <= 64");
        const uint32_t Ll = p->L_local ? p->L_local : p->L;
        if (Ll > 8192) return fail(PANNS_EINVAL, "search: L_local > 8192 is not supported");
    }
    if (p->warps_per_block > 8) return fail(PANNS_EINVAL, "search: warps_per_block must be <= 8");
    if (p->flags & ~(PANNS_FLAG_CUDA_GRAPH | PANNS_FLAG_LEARNED)) return fail(PANNS_EINVAL, "search: unknown flags");
    if (p->flags & PANNS_FLAG_LEARNED) {
        if (!h->has_mlp) return fail(PANNS_ESTATE, "search: PANNS_FLAG_LEARNED without a network (panns_set_learned)");
        const bool ok = p->mode == PANNS_MODE_NSG_SEQ || p->mode == PANNS_MODE_TOP_M ||
                        (p->mode == PANNS_MODE_PSS_V5 && p->T == 1);
        if (!ok) return fail(PANNS_EINVAL, "search: PANNS_FLAG_LEARNED is for NSG_SEQ, TOP_M and PSS_V5 at T = 1");
    }
    if (p->L_query && p->mode == PANNS_MODE_PSS_V5 && p->T > 1)
        return fail(PANNS_EINVAL, "search: L_query is not supported by PSS_V5 with T > 1");
    if (p->storage > PANNS_STORE_FP8) return fail(PANNS_EINVAL, "search: unknown storage");
    if (p->warps_per_query > 1) {
        if (p->warps_per_query != 2 && p->warps_per_query != 4 && p->warps_per_query != 8)
            return fail(PANNS_EINVAL, "search: warps_per_query must be 0, 1, 2, 4 or 8");
        const bool ok = p->mode == PANNS_MODE_NSG_SEQ || p->mode == PANNS_MODE_TOP_M ||
                        (p->mode == PANNS_MODE_PSS_V5 && p->T == 1);
        if (!ok)
            return fail(PANNS_EINVAL, "search: warps_per_query > 1 is for NSG_SEQ, TOP_M and PSS_V5 at T = 1");
        if (h->max_deg > (uint32_t) kBuf)
            return fail(PANNS_EINVAL, "search: warps_per_query > 1 needs a graph degree <= " + std::to_string(kBuf));
    }
    if (p->storage != PANNS_STORE_FP32) {
        if (p->storage != h->storage)
            return fail(PANNS_EINVAL, "search: that reduced copy was not built (panns_set_base storage)");
        const bool ok = p->mode == PANNS_MODE_NSG_SEQ || p->mode == PANNS_MODE_TOP_M ||
                        (p->mode == PANNS_MODE_PSS_V5 && p->T == 1);
        if (!ok) return fail(PANNS_EINVAL, "search: reduced storage is for NSG_SEQ and TOP_M");
    }
    return PANNS_OK;
}

}  // namespace

// Preferred shared-memory carveout (percent of the SM's 228 KB) for
// `blocks` resident blocks of `smem` dynamic bytes each (1 KB reserved per
// block); -1 (the driver's choice) when blocks is 0.
static int carveout_percent(size_t smem, uint32_t blocks) {
    if (!blocks) return -1;
    const size_t need = (size_t) blocks * (smem + 1024);
    const size_t total = 228u * 1024u;
    return (int) std::min<size_t>(100, (need * 100 + total - 1) / total);
}

// What one search launch enqueues: two 4-byte memsets, the optional layout of
// row-major device queries, and the kernel.
struct LaunchDesc {
    const void *kern;
    uint32_t blocks, threads;
    size_t smem;
    const void *args;       // SearchArgs or PssArgs
    size_t args_size;
    uint32_t *counter, *error;
    const float *rows;      // row-major queries to lay out into rows_cm (or null)
    float *rows_cm;
    uint32_t rows_n, d, dpad;
    // Learned decisions computed before the search (mlp_decide), or mlp null.
    const MlpDev *mlp;
    const float *mlp_q;     // chain-major queries
    uint32_t mlp_nq, mlp_L, mlp_K;
    const uint32_t *mlp_Lq;
    MlpScratch mlp_scratch;
    uint32_t *mlp_record;
};

static cudaError_t enqueue_plain(const LaunchDesc &l, int num_sms, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(l.counter, 0, 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(l.error, 0, 4, s);
    if (e == cudaSuccess && l.rows) {
        const uint64_t total = (uint64_t) l.rows_n * l.dpad;
        const int pb = (int) std::min<uint64_t>((total + 255) / 256, (uint64_t) num_sms * 32);
        permute_rows_kernel<<<std::max(pb, 1), 256, 0, s>>>(l.rows, l.rows_cm, l.rows_n, (int) l.d,
                                                             (int) l.dpad, nullptr);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && l.mlp)
        e = mlp_decide(*l.mlp, l.mlp_q, l.dpad, l.mlp_nq, l.mlp_L, l.mlp_Lq, l.mlp_K, l.mlp_scratch, l.mlp_record, s);
    if (e == cudaSuccess) {
        void *argv[] = {const_cast<void *>(l.args)};
        e = cudaLaunchKernel(l.kern, dim3(l.blocks), dim3(l.threads), argv, l.smem, s);
    }
    return e;
}

// Enqueue directly, or (graph) replay the handle's captured graph of the same
// sequence, re-capturing and updating it in place when the key changed.
static int enqueue_launch(panns_index *h, const LaunchDesc &l, cudaStream_t s, bool graph) {
    if (!graph) {
        CU(enqueue_plain(l, h->num_sms, s));
        return PANNS_OK;
    }
    std::vector<uint8_t> key;
    auto put = [&key](const void *v, size_t n) {
        key.insert(key.end(), (const uint8_t *) v, (const uint8_t *) v + n);
    };
    const uint64_t f[] = {(uint64_t) (uintptr_t) l.kern, l.blocks, l.threads, l.smem,
                          (uint64_t) (uintptr_t) l.counter, (uint64_t) (uintptr_t) l.error,
                          (uint64_t) (uintptr_t) l.rows, (uint64_t) (uintptr_t) l.rows_cm,
                          l.rows_n, l.d, l.dpad,
                          (uint64_t) (uintptr_t) l.mlp, (uint64_t) (uintptr_t) l.mlp_q, l.mlp_nq, l.mlp_L, l.mlp_K,
                          (uint64_t) (uintptr_t) l.mlp_Lq, (uint64_t) (uintptr_t) l.mlp_scratch.X,
                          (uint64_t) (uintptr_t) l.mlp_scratch.H1, (uint64_t) (uintptr_t) l.mlp_scratch.H2,
                          (uint64_t) (uintptr_t) l.mlp_scratch.Z, l.mlp_scratch.rows,
                          (uint64_t) (uintptr_t) l.mlp_record};
    put(f, sizeof(f));
    if (l.mlp) put(l.mlp, sizeof(MlpDev));  // value-initialised, so padding compares equal
    put(l.args, l.args_size);  // zero-filled structs, so padding compares equal
    if (!h->gexec || key != h->gkey) {
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        const cudaError_t e = enqueue_plain(l, h->num_sms, s);
        const cudaError_t e2 = cudaStreamEndCapture(s, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            CU(e != cudaSuccess ? e : e2);
        }
        bool updated = false;
        if (h->gexec) {
            cudaGraphExecUpdateResultInfo info;
            updated = cudaGraphExecUpdate(h->gexec, g, &info) == cudaSuccess;
            if (!updated) {
                cudaGetLastError();
                cudaGraphExecDestroy(h->gexec);
                h->gexec = nullptr;
            }
        }
        if (!updated) {
            const cudaError_t ei = cudaGraphInstantiate(&h->gexec, g, 0);
            if (ei != cudaSuccess) {
                cudaGraphDestroy(g);
                h->gexec = nullptr;
                CU(ei);
            }
        }
        cudaGraphDestroy(g);
        h->gkey.swap(key);
    }
    CU(cudaGraphLaunch(h->gexec, s));
    return PANNS_OK;
}

// Launch the search for nq device queries (chain-major at d_queries_cm; when
// d_rows is set they are first laid out there from row-major d_rows), with
// device init ids and optional per-query queue lengths; everything enqueued
// on `stream`.
static int launch_search(panns_index *h, const panns_search_params *p, float *d_queries_cm,
                         const float *d_rows, uint32_t nq, const uint32_t *d_init, uint32_t init_stride,
                         const uint32_t *d_lq, uint32_t *d_out, uint4 *d_stats, cudaStream_t stream,
                         bool time_it) {
    const int CL = (int) (h->dpad / 32);
    const uint32_t order = p->mode == PANNS_MODE_EFANNA ? ORDER_EFANNA : ORDER_PANNS;
    const uint32_t kind = p->distance == PANNS_DIST_L2 ? KIND_L2 : KIND_IP;
    const bool pss = p->mode == PANNS_MODE_PSS_V5 && p->T > 1;
    uint32_t wpq = p->warps_per_query > 1 ? p->warps_per_query : 1u;
    if (p->warps_per_query == 0 && p->warps_per_block == 0 && p->blocks_per_sm == 0 &&
        (p->mode == PANNS_MODE_NSG_SEQ || p->mode == PANNS_MODE_TOP_M || (p->mode == PANNS_MODE_PSS_V5 && p->T == 1)) &&
        h->max_deg <= (uint32_t) kBuf) {
        // Automatic block shape (same ids either way), from the 1M x 96 and
        // 1M x 128 measurements: 8 warps per query up to one query per SM and
        // for queues of 2048 and more, 2 up to ten queries per SM, else one.
        const uint32_t sms = (uint32_t) h->num_sms;
        if (p->L >= 2048 || nq <= sms) wpq = 8;
        else if (nq <= 10 * sms) wpq = 2;
    }
    const void *kern = wpq > 1 ? search_block_kernel_ptr(kind, CL, wpq, p->storage)
                               : pss ? pss_kernel_ptr(kind, CL) : search_kernel_ptr(kind, order, CL, p->storage);
    if (!kern) return fail(PANNS_EINVAL, "search: unsupported dimension");
    const uint32_t M = p->mode == PANNS_MODE_TOP_M ? p->M : 1u;
    const uint32_t qcap = ((p->L + 31) / 32) * 32;
    const uint32_t L_local = p->L_local ? p->L_local : p->L;
    const uint32_t wcap = ((L_local + 31) / 32) * 32;
    // Block shape: wpb queries of one warp each, or one query of wpq warps.
    uint32_t wpb = wpq > 1 ? wpq : (p->warps_per_block ? p->warps_per_block : 4u);
    size_t per_warp = pss ? pss_smem_bytes(qcap, p->T, wcap) : warp_smem_bytes(qcap);
    if (pss && !p->warps_per_block) {
        while (wpb > 1 && wpb * per_warp > (100u << 10)) --wpb;
    }
    if (wpq == 1 && !p->warps_per_block) {  // default block shape: as many warps as fit (long queues)
        while (wpb > 1 && wpb * per_warp > (227u << 10)) --wpb;
    }
    if (per_warp > (227u << 10))
        return fail(PANNS_EINVAL, "search: the queues (L, T x L_local) do not fit in shared memory");
    const size_t smem = wpq > 1 ? (size_t) block_smem_bytes(qcap, wpq) : (size_t) wpb * per_warp;
    if (smem > (227u << 10)) return fail(PANNS_EINVAL, "search: the queue does not fit in shared memory");
    const uint32_t qpb = wpq > 1 ? 1u : wpb;  // queries in flight per block
    {
        cudaFuncAttributes fa;
        CU(cudaFuncGetAttributes(&fa, kern));
        if ((int) (wpb * 32) > fa.maxThreadsPerBlock)
            return fail(PANNS_EINVAL, "search: warps_per_block must be <= " + std::to_string(fa.maxThreadsPerBlock / 32) +
                                          " for this kernel");
    }
    CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    // The L1 / shared-memory split: the driver's first (enough shared memory
    // for the most resident blocks); with a block count (blocks_per_sm, or the
    // default below), just enough shared memory for that many blocks, the rest
    // of the array left to L1, which caches the gathered rows.
    CU(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                            carveout_percent(smem, p->blocks_per_sm)));
    int per_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int) wpb * 32, smem));
    if (per_sm < 1) return fail(PANNS_EINVAL, "search: L too large for shared memory");
    uint32_t bps = p->blocks_per_sm;
    if (!bps) {
        // As many resident blocks as fit, unless that takes the whole 228 KB
        // array as shared memory (28 KB of L1 left): then as many as fit in
        // 196 KB. Measured on the 1M set: L = 448, 8.9 ms (5 blocks) against
        // 10.0 ms (6 blocks); L = 512 with 2-warp blocks, 9.8 ms (10) against 11.0 (12).
        const size_t per_block = smem + 1024;
        const int fit = (int) ((196u << 10) / per_block);
        if ((size_t) per_sm * per_block > (196u << 10) && fit >= 1) bps = (uint32_t) fit;
    }
    if (bps) {
        CU(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, carveout_percent(smem, bps)));
        per_sm = std::min(per_sm, (int) bps);
    }
    uint32_t blocks = (uint32_t) per_sm * (uint32_t) h->num_sms;
    const uint32_t need_blocks = (nq + qpb - 1) / qpb;
    blocks = std::max(1u, std::min(blocks, need_blocks));
    // Per-slot visited bitsets and dirty-word lists. When they must grow, they
    // may take what they already hold plus half of the device's free memory
    // (at least 1 GiB): at N = 100M a slot is 12.5 MB, and the 3,552 resident
    // warps of a 148-SM part need 44 GB, which a 180 GB B200 holding the
    // 100M index (about 77 GB) still has.
    const uint32_t vis_words = (h->n + 31) / 32;
    const uint32_t dirty_cap = 8192;
    const uint64_t per_slot = ((uint64_t) vis_words + dirty_cap) * 4;
    if ((uint64_t) blocks * qpb > h->vis_slots || h->vis_words != vis_words) {
        size_t free_b = 0, total_b = 0;
        CU(cudaMemGetInfo(&free_b, &total_b));
        const uint64_t held = ((uint64_t) h->visited.n + h->dirty.n) * 4;
        const uint64_t budget = std::max<uint64_t>(1ull << 30, held + free_b / 2);
        const uint64_t max_slots = budget / per_slot;
        if ((uint64_t) blocks * qpb > max_slots) blocks = (uint32_t) std::max<uint64_t>(1, max_slots / qpb);
    }
    const uint32_t nslots = blocks * qpb;
    if (h->vis_slots < nslots || h->vis_words != vis_words) {
        CU(h->visited.ensure((size_t) nslots * vis_words));
        CU(cudaMemsetAsync(h->visited.p, 0, (size_t) nslots * vis_words * 4, stream));
        CU(h->dirty.ensure((size_t) nslots * dirty_cap));
        h->vis_slots = nslots;
        h->vis_words = vis_words;
    }
    CU(h->counter.ensure(1));
    CU(h->error.ensure(1));
    const bool learned = (p->flags & PANNS_FLAG_LEARNED) != 0;
    if (learned) {
        // Scratch of the batched inference (chunks of up to 16,384 queries)
        // and the per-query decision records, sized before any capture.
        const uint32_t chunk = std::min<uint32_t>(nq, 16384);
        if (h->mlp_chunk < chunk || h->mlp_scratch.n < (size_t) h->mlp_chunk * (h->d + 2u * kMlpH + h->mlp.R)) {
            const uint32_t c = std::max(chunk, h->mlp_chunk);
            CU(h->mlp_scratch.ensure((size_t) c * (h->d + 2u * kMlpH + h->mlp.R)));
            h->mlp_chunk = c;
        }
        if (h->mlp_rec_cap < nq) {
            CU(h->mlp_record.ensure((size_t) nq * kMlpRecWords));
            h->mlp_rec_cap = nq;
        }
        h->mlp_last_nq = nq;
    }
    SearchArgs a;
    memset(&a, 0, sizeof(a));
    a.decisions = learned ? h->mlp_record.p : nullptr;
    a.dec_L_init = h->mlp.L_init;
    a.vec = reinterpret_cast<const float4 *>(h->vec.p);
    a.norms = h->norms.p;
    a.head = h->head.p;
    a.ovf_off = h->ovf_off.p;
    a.ovf = h->ovf.p;
    a.orig = h->orig.p;
    a.vec_lo = h->vec_lo.p;
    a.norms_lo = h->norms_lo.p;
    a.scales = h->scales.p;
    a.d = h->d;
    a.n = h->n;
    a.queries = reinterpret_cast<const float4 *>(d_queries_cm);
    a.nq = nq;
    a.init_ids = d_init;
    a.init_stride = init_stride;
    a.K = p->K;
    a.L = p->L;
    a.Lq = d_lq;
    a.M = M;
    a.out_ids = d_out;
    a.out_stats = d_stats;
    a.visited = h->visited.p;
    a.vis_words = vis_words;
    a.dirty = h->dirty.p;
    a.dirty_cap = dirty_cap;
    a.counter = h->counter.p;
    a.error = h->error.p;
    a.queue_cap = qcap;
    // Block kernel: candidates per warp and merge round, so that a warp's
    // fresh neighbours (at most max_deg per candidate) fit its list.
    a.block_round = std::max(1u, std::min<uint32_t>(kCandGroup, kBuf / std::max(1u, h->max_deg)));
    PssArgs pa;
    memset(&pa, 0, sizeof(pa));
    memcpy(&pa.s, &a, sizeof(a));
    pa.T = p->T;
    pa.L_local = L_local;
    pa.X = p->X;
    pa.wcap = wcap;
    LaunchDesc l;
    memset(&l, 0, sizeof(l));
    l.kern = kern;
    l.blocks = blocks;
    l.threads = wpb * 32;
    l.smem = smem;
    l.args = pss ? (const void *) &pa : (const void *) &a;
    l.args_size = pss ? sizeof(pa) : sizeof(a);
    l.counter = h->counter.p;
    l.error = h->error.p;
    l.rows = d_rows;
    l.rows_cm = d_queries_cm;
    l.rows_n = nq;
    l.d = h->d;
    l.dpad = h->dpad;
    if (learned) {
        l.mlp = &h->mlp;
        l.mlp_q = d_queries_cm;
        l.mlp_nq = nq;
        l.mlp_L = p->L;
        l.mlp_K = p->K;
        l.mlp_Lq = d_lq;
        float *sp = h->mlp_scratch.p;
        const size_t c = h->mlp_chunk;
        l.mlp_scratch = MlpScratch{sp, sp + c * h->d, sp + c * (h->d + kMlpH), sp + c * (h->d + 2u * kMlpH),
                                   h->mlp_chunk};
        l.mlp_record = h->mlp_record.p;
    }
    if (time_it) CU(cudaEventRecord(h->ev0, stream));
    int rc = enqueue_launch(h, l, stream, (p->flags & PANNS_FLAG_CUDA_GRAPH) != 0);
    if (rc) return rc;
    if (time_it) CU(cudaEventRecord(h->ev1, stream));
    return PANNS_OK;
}

// Init ids as device ids on the device: the caller's (validated: in range,
// distinct per list), efanna2e's per-query random lists, or the default PANNS
// list, which is built once per (layout, L) and kept on the device.
static int stage_init(panns_index *h, const panns_search_params *p, const uint32_t *init_ids,
                      uint32_t nq, cudaStream_t stream, const uint32_t *&d_init, uint32_t &stride) {
    const uint32_t L = p->L;
    const bool efanna = p->mode == PANNS_MODE_EFANNA;
    stride = efanna ? L : 0;
    if (!efanna && !init_ids && h->init_def_L == L) {
        d_init = h->init_def.p;
        return PANNS_OK;
    }
    std::vector<uint32_t> buf;
    const uint32_t *ids = init_ids;
    if (!ids) {
        if (efanna) {
            int32_t st[40];
            panns_rand_seed(st, 1);
            buf.resize((size_t) nq * L);
            int rc = panns_efanna_init_ids(h, L, nq, st, buf.data());
            if (rc) return rc;
        } else {
            buf.resize(L);
            int rc = panns_prepare_init_ids(h, L, buf.data());
            if (rc) return rc;
        }
        ids = buf.data();
    }
    // Valid, distinct vertices per list; handed over as device ids in the same order.
    const uint32_t groups = efanna ? nq : 1;
    std::vector<uint32_t> dev((size_t) groups * L);
    const bool by_sort = (uint64_t) groups * L * 16 < h->n;
    std::vector<uint8_t> seen(by_sort ? 0 : h->n, 0);
    std::vector<uint32_t> tmp;
    for (uint32_t g = 0; g < groups; ++g) {
        const uint32_t *x = ids + (size_t) g * L;
        for (uint32_t i = 0; i < L; ++i) {
            if (x[i] >= h->n) return fail(PANNS_EINVAL, "search: init id out of range");
            dev[(size_t) g * L + i] = h->inv[x[i]];
        }
        if (by_sort) {
            tmp.assign(x, x + L);
            std::sort(tmp.begin(), tmp.end());
            if (std::adjacent_find(tmp.begin(), tmp.end()) != tmp.end())
                return fail(PANNS_EINVAL, "search: duplicate init id");
        } else {
            for (uint32_t i = 0; i < L; ++i) {
                if (seen[x[i]]) return fail(PANNS_EINVAL, "search: duplicate init id");
                seen[x[i]] = 1;
            }
            for (uint32_t i = 0; i < L; ++i) seen[x[i]] = 0;
        }
    }
    if (!efanna && !init_ids) {
        CU(h->init_def.ensure(L));
        // Ordered on the launch stream (the source is staged before the call returns).
        CU(cudaMemcpyAsync(h->init_def.p, dev.data(), (size_t) L * 4, cudaMemcpyHostToDevice, stream));
        h->init_def_L = L;
        d_init = h->init_def.p;
        return PANNS_OK;
    }
    CU(h->init.ensure(dev.size()));
    CU(cudaMemcpyAsync(h->init.p, dev.data(), dev.size() * 4, cudaMemcpyHostToDevice, stream));
    d_init = h->init.p;
    return PANNS_OK;
}

// Per-query queue lengths (validated K <= L_query[i] <= L) on the device, or null.
static int stage_lq(panns_index *h, const panns_search_params *p, uint32_t nq, cudaStream_t stream,
                    const uint32_t *&d_lq) {
    d_lq = nullptr;
    if (!p->L_query) return PANNS_OK;
    for (uint32_t i = 0; i < nq; ++i)
        if (p->L_query[i] < p->K || p->L_query[i] > p->L)
            return fail(PANNS_EINVAL, "search: need K <= L_query[i] <= L");
    CU(h->lq.ensure(nq));
    CU(cudaMemcpyAsync(h->lq.p, p->L_query, (size_t) nq * 4, cudaMemcpyHostToDevice, stream));
    d_lq = h->lq.p;
    return PANNS_OK;
}

static int finish(panns_index *h, uint32_t nq, uint32_t K, uint32_t *out_ids, panns_stats *stats,
                  double t0_ms) {
    h->h_stats.resize(nq);
    uint32_t err = 0;
    CU(cudaMemcpyAsync(out_ids, h->out.p, (size_t) nq * K * 4, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaMemcpyAsync(h->h_stats.data(), h->stats.p, (size_t) nq * sizeof(uint4), cudaMemcpyDeviceToHost,
                       h->stream));
    CU(cudaMemcpyAsync(&err, h->error.p, 4, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    if (err & ERR_BAD_ID) return fail(PANNS_EDEVICE, "search: the graph holds a neighbour id >= N");
    if (err & ERR_BAD_INIT) return fail(PANNS_EDEVICE, "search: init id >= N");
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        for (const uint4 &s : h->h_stats) {
            stats->n_dist += s.x;
            stats->n_expand += s.y;
            stats->n_edges += s.z;
            stats->n_iter += s.w;
        }
        float ms = 0.f;
        CU(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        stats->kernel_ms = ms;
        const double t1 = std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now().time_since_epoch()).count();
        stats->total_ms = t1 - t0_ms;
    }
    return PANNS_OK;
}

static double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

extern "C" {

int panns_search(panns_index *h, const panns_search_params *p, const uint32_t *init_ids,
                 uint32_t q_begin, uint32_t nq, uint32_t *out_ids, panns_stats *stats) {
    if (!h) return fail(PANNS_EINVAL, "panns_search: NULL handle");
    const double t0 = now_ms();
    int rc = check_params(h, p);
    if (rc) return rc;
    if (!out_ids && nq) return fail(PANNS_EINVAL, "panns_search: NULL out_ids");
    if ((uint64_t) q_begin + nq > h->nq) return fail(PANNS_EINVAL, "panns_search: query range out of bounds");
    if (nq == 0) {
        if (stats) memset(stats, 0, sizeof(*stats));
        return PANNS_OK;
    }
    CU(cudaSetDevice(h->device));
    const uint32_t *d_init = nullptr, *d_lq = nullptr;
    uint32_t stride = 0;
    rc = stage_init(h, p, init_ids, nq, h->stream, d_init, stride);
    if (!rc) rc = stage_lq(h, p, nq, h->stream, d_lq);
    if (rc) return rc;
    CU(h->out.ensure((size_t) nq * p->K));
    CU(h->stats.ensure(nq));
    rc = launch_search(h, p, h->queries.p + (size_t) q_begin * h->dpad, nullptr, nq, d_init, stride, d_lq,
                       h->out.p, h->stats.p, h->stream, true);
    if (rc) return rc;
    return finish(h, nq, p->K, out_ids, stats, t0);
}

int panns_search_host(panns_index *h, const panns_search_params *p, const float *queries, uint32_t nq,
                      const uint32_t *init_ids, uint32_t *out_ids, panns_stats *stats) {
    if (!h) return fail(PANNS_EINVAL, "panns_search_host: NULL handle");
    const double t0 = now_ms();
    int rc = check_params(h, p);
    if (rc) return rc;
    if (nq == 0) {
        if (stats) memset(stats, 0, sizeof(*stats));
        return PANNS_OK;
    }
    if (!queries || !out_ids) return fail(PANNS_EINVAL, "panns_search_host: NULL argument");
    CU(cudaSetDevice(h->device));
    const uint32_t *d_init = nullptr, *d_lq = nullptr;
    uint32_t stride = 0;
    rc = stage_init(h, p, init_ids, nq, h->stream, d_init, stride);
    if (!rc) rc = stage_lq(h, p, nq, h->stream, d_lq);
    if (rc) return rc;
    // Rows go up as they are; the chain-major layout is part of the launch.
    CU(h->raw.ensure((size_t) nq * h->d));
    CU(h->hq.ensure((size_t) nq * h->dpad));
    CU(cudaMemcpyAsync(h->raw.p, queries, (size_t) nq * h->d * sizeof(float), cudaMemcpyHostToDevice,
                       h->stream));
    CU(h->out.ensure((size_t) nq * p->K));
    CU(h->stats.ensure(nq));
    rc = launch_search(h, p, h->hq.p, h->raw.p, nq, d_init, stride, d_lq, h->out.p, h->stats.p, h->stream,
                       true);
    if (rc) return rc;
    return finish(h, nq, p->K, out_ids, stats, t0);
}

int panns_search_device(panns_index *h, const panns_search_params *p, const float *d_queries,
                        uint32_t nq, const uint32_t *init_ids, uint32_t *d_out_ids, void *stream,
                        panns_stats *stats) {
    if (!h) return fail(PANNS_EINVAL, "panns_search_device: NULL handle");
    int rc = check_params(h, p);
    if (rc) return rc;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (nq == 0) return PANNS_OK;
    if (!d_queries || !d_out_ids) return fail(PANNS_EINVAL, "panns_search_device: NULL argument");
    CU(cudaSetDevice(h->device));
    cudaStream_t st = stream ? (cudaStream_t) stream : h->stream;
    const uint32_t *d_init = nullptr, *d_lq = nullptr;
    uint32_t stride = 0;
    rc = stage_init(h, p, init_ids, nq, st, d_init, stride);
    if (!rc) rc = stage_lq(h, p, nq, st, d_lq);
    if (rc) return rc;
    CU(h->dq.ensure((size_t) nq * h->dpad));
    return launch_search(h, p, h->dq.p, d_queries, nq, d_init, stride, d_lq, d_out_ids, nullptr, st, false);
}

int panns_ground_truth(panns_index *h, const float *queries, uint32_t nq, uint32_t k, uint32_t *out_ids,
                       double *out_dist) {
    if (!h || (nq && (!queries || !out_ids))) return fail(PANNS_EINVAL, "panns_ground_truth: NULL argument");
    if (nq == 0) return PANNS_OK;
    int rc = finalize(h);
    if (rc) return rc;
    if (k == 0 || k > h->n) return fail(PANNS_EINVAL, "panns_ground_truth: need 0 < k <= N");
    CU(cudaSetDevice(h->device));
    // 1. An upper bound per query: a top-M search for k results (exact FP32),
    // with a queue that also holds every neighbour of the entry (the PANNS
    // init list), so graphs whose parts meet only at the entry are covered.
    panns_search_params p{};
    p.mode = PANNS_MODE_TOP_M;
    p.distance = PANNS_DIST_L2;
    p.K = k;
    p.L = std::min(h->n, std::max(std::max(2 * k, 256u), std::min(h->max_deg + 2 * k, 8192u)));
    p.M = 8;
    p.T = 1;
    p.X = 1;
    std::vector<uint32_t> sids((size_t) nq * k);
    rc = panns_search_host(h, &p, queries, nq, nullptr, sids.data(), nullptr);
    if (rc) return rc;
    DevBuf<float> dq;
    DevBuf<uint32_t> dids, dcnt;
    DevBuf<double> dtau;
    CU(dq.ensure((size_t) nq * h->d));
    CU(dids.ensure((size_t) nq * k));
    CU(dtau.ensure(nq));
    CU(dcnt.ensure(nq));
    CU(cudaMemcpyAsync(dq.p, queries, (size_t) nq * h->d * 4, cudaMemcpyHostToDevice, h->stream));
    CU(cudaMemcpyAsync(dids.p, sids.data(), (size_t) nq * k * 4, cudaMemcpyHostToDevice, h->stream));
    gt_tau_kernel<<<(nq + 3) / 4, 128, 0, h->stream>>>(h->base_raw.p, (int) h->d, dq.p, nq, dids.p, k, dtau.p);
    CU(cudaGetLastError());
    // 2. Collect every vertex within the bound. A pass scans all vertices for
    // a set of queries with lists of `cap` entries (counts go on past cap).
    const uint32_t vt = (h->n + kGtV - 1) / kGtV;
    auto collect = [&](const float *qrows, const double *tau, uint32_t m, uint32_t cap, uint32_t *dc, double *cd,
                       uint32_t *ci) -> cudaError_t {
        cudaError_t e = cudaMemsetAsync(dc, 0, m * 4ull, h->stream);
        for (uint32_t t0 = 0; e == cudaSuccess && t0 < vt; t0 += 65535u) {
            dim3 grid((m + kGtQ - 1) / kGtQ, std::min(65535u, vt - t0));
            gt_collect_kernel<<<grid, 256, 0, h->stream>>>(h->base_raw.p, h->n, (int) h->d, qrows, m, tau, cap, dc,
                                                           cd, ci, t0);
            e = cudaGetLastError();
        }
        return e;
    };
    // The exact (distance, id) order of one query's list; the first k are the answer.
    std::vector<std::pair<double, uint32_t>> tmp;
    auto finish = [&](uint32_t q, const double *ld, const uint32_t *li, uint32_t c) -> int {
        if (c < k) return fail(PANNS_EDEVICE, "panns_ground_truth: fewer candidates than k");
        tmp.resize(c);
        for (uint32_t i = 0; i < c; ++i) tmp[i] = {ld[i], li[i]};
        std::partial_sort(tmp.begin(), tmp.begin() + k, tmp.end());
        for (uint32_t i = 0; i < k; ++i) {
            out_ids[(size_t) q * k + i] = tmp[i].second;
            if (out_dist) out_dist[(size_t) q * k + i] = tmp[i].first;
        }
        return PANNS_OK;
    };
    const uint32_t cap = std::max(4 * k, 64u);
    std::vector<uint32_t> cnt(nq);
    std::vector<uint32_t> over;  // queries whose lists overflowed
    {
        DevBuf<double> cd;
        DevBuf<uint32_t> ci;
        CU(cd.ensure((size_t) nq * cap));
        CU(ci.ensure((size_t) nq * cap));
        CU(collect(dq.p, dtau.p, nq, cap, dcnt.p, cd.p, ci.p));
        CU(cudaMemcpyAsync(cnt.data(), dcnt.p, nq * 4ull, cudaMemcpyDeviceToHost, h->stream));
        std::vector<double> hd((size_t) nq * cap);
        std::vector<uint32_t> hi((size_t) nq * cap);
        CU(cudaMemcpyAsync(hd.data(), cd.p, hd.size() * 8, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaMemcpyAsync(hi.data(), ci.p, hi.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
        for (uint32_t q = 0; q < nq; ++q) {
            if (cnt[q] > cap) {
                over.push_back(q);
                continue;
            }
            rc = finish(q, hd.data() + (size_t) q * cap, hi.data() + (size_t) q * cap, cnt[q]);
            if (rc) return rc;
        }
    }
    // 3. Queries whose bound was loose (the search missed their part of the
    // graph): again, a few at a time, each list as long as its count, within
    // 4 GiB of lists per pass.
    const size_t budget = 4ull << 30;
    for (size_t g0 = 0; g0 < over.size();) {
        size_t g1 = g0;
        uint32_t gcap = 0;
        while (g1 < over.size()) {
            const uint32_t c2 = std::max(gcap, cnt[over[g1]]);
            if (g1 > g0 && (size_t) (g1 - g0 + 1) * c2 * 12 > budget) break;
            gcap = c2;
            ++g1;
        }
        const uint32_t m = (uint32_t) (g1 - g0);
        if ((size_t) m * gcap * 12 > budget)
            return fail(PANNS_ENOMEM, "panns_ground_truth: a query's bound holds " + std::to_string(gcap) +
                                          " vertices, more than the 4 GiB of candidate lists allowed");
        std::vector<float> qh((size_t) m * h->d);
        std::vector<double> th(m);
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t q = over[g0 + i];
            std::copy(queries + (size_t) q * h->d, queries + (size_t) (q + 1) * h->d, qh.begin() + (size_t) i * h->d);
        }
        DevBuf<float> gq;
        DevBuf<double> gt, cd;
        DevBuf<uint32_t> gc, ci;
        CU(gq.ensure(qh.size()));
        CU(gt.ensure(m));
        CU(gc.ensure(m));
        CU(cd.ensure((size_t) m * gcap));
        CU(ci.ensure((size_t) m * gcap));
        CU(cudaMemcpyAsync(gq.p, qh.data(), qh.size() * 4, cudaMemcpyHostToDevice, h->stream));
        for (uint32_t i = 0; i < m; ++i)
            CU(cudaMemcpyAsync(gt.p + i, dtau.p + over[g0 + i], 8, cudaMemcpyDeviceToDevice, h->stream));
        CU(collect(gq.p, gt.p, m, gcap, gc.p, cd.p, ci.p));
        std::vector<uint32_t> c2(m);
        std::vector<double> hd((size_t) m * gcap);
        std::vector<uint32_t> hi((size_t) m * gcap);
        CU(cudaMemcpyAsync(c2.data(), gc.p, m * 4ull, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaMemcpyAsync(hd.data(), cd.p, hd.size() * 8, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaMemcpyAsync(hi.data(), ci.p, hi.size() * 4, cudaMemcpyDeviceToHost, h->stream));
        CU(cudaStreamSynchronize(h->stream));
        for (uint32_t i = 0; i < m; ++i) {
            if (c2[i] > gcap) return fail(PANNS_EDEVICE, "panns_ground_truth: candidate count changed between passes");
            rc = finish(over[g0 + i], hd.data() + (size_t) i * gcap, hi.data() + (size_t) i * gcap, c2[i]);
            if (rc) return rc;
        }
        g0 = g1;
    }
    return PANNS_OK;
}

int panns_recall(const uint32_t *result_ids, uint32_t nq, uint32_t K, const uint32_t *true_ids,
                 uint32_t true_k, uint32_t L, uint32_t at, double *out) {
    if (!result_ids || !true_ids || !out) return fail(PANNS_EINVAL, "panns_recall: NULL argument");
    if (at == 0 || at > true_k || at > 100) return fail(PANNS_EINVAL, "panns_recall: bad k");
    if (nq == 0) {
        *out = 0.0;
        return PANNS_OK;
    }
    const uint32_t prefix = std::min(std::min(L, 100u), std::min(K, at));
    double hits = 0;
    for (uint32_t q = 0; q < nq; ++q) {
        const uint32_t *t = true_ids + (size_t) q * true_k;
        const uint32_t *r = result_ids + (size_t) q * K;
        for (uint32_t i = 0; i < at; ++i)
            for (uint32_t j = 0; j < prefix; ++j)
                if (r[j] == t[i]) {
                    hits += 1;
                    break;
                }
    }
    *out = hits / ((double) at * nq);
    return PANNS_OK;
}

int panns_load_true_nn(const char *path, uint32_t *nq, uint32_t *K, uint32_t *ids, float *dists) {
    if (!path || !nq || !K) return fail(PANNS_EINVAL, "panns_load_true_nn: NULL argument");
    FILE *f = fopen(path, "rb");
    if (!f) return fail(PANNS_EIO, std::string("cannot open ") + path);
    uint32_t hdr[2];
    if (fread(hdr, 4, 2, f) != 2) {
        fclose(f);
        return fail(PANNS_EIO, "truncated true-NN header");
    }
    *nq = hdr[0];
    *K = hdr[1];
    if (!ids) {
        fclose(f);
        return PANNS_OK;
    }
    std::vector<uint32_t> rec(2ull * hdr[1]);
    for (uint32_t q = 0; q < hdr[0]; ++q) {
        if (fread(rec.data(), 4, rec.size(), f) != rec.size()) {
            fclose(f);
            return fail(PANNS_EIO, "truncated true-NN body");
        }
        for (uint32_t i = 0; i < hdr[1]; ++i) {
            ids[(size_t) q * hdr[1] + i] = rec[2 * i];
            if (dists) memcpy(dists + (size_t) q * hdr[1] + i, &rec[2 * i + 1], 4);
        }
    }
    fclose(f);
    return PANNS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// panns_search_static: the batched search without any memory allocation.
//
// Some callers cannot allocate GPU memory at search time: a server that
// reserves all device memory for a framework's own pool at start-up, a
// real-time loop where an allocation (and the device-wide synchronisation a
// cudaFree implies) would break its latency budget, or a plug-in loaded into
// a host process that forbids allocations after initialisation. For them this
// entry point takes its scratch — the per-warp visited bitsets and cleared-word
// lists, the work counter, the error word, the chain-major copy of the
// queries and the init ids — from one fixed array of kStaticScratchBytes that
// lives in the library's device image. Every GPU that loads the library holds
// that array until the process exits.
//
// The first call on a device looks up the array's device address
// (cudaGetSymbolAddress). No call may be made while a stream is being
// captured: every call copies the init list from host memory, reads the
// error word back and synchronises its stream before it returns.
// All calls share the array and it keeps the last call's contents: each call
// zeroes what must start at zero. Calls that overlap on the GPU (from two
// threads, or on two streams) race on the array and must not be made.
// ---------------------------------------------------------------------------
#include <mutex>

namespace {

constexpr size_t kStaticScratchBytes = 32ull << 20;   // 32 MiB
constexpr uint32_t kStaticMaxL = 1024;               // init ids held in the array
constexpr uint32_t kStaticDirtyCap = 2048;           // cleared-word list per warp
constexpr size_t kStaticHeader = 256;                // counter, error

static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

std::mutex g_static_mu;
void *g_static_addr[64] = {nullptr};

int static_scratch_address(int device, unsigned char **out) {
    if (device < 0 || device >= 64) return fail(PANNS_EINVAL, "panns_search_static: device index >= 64");
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(PANNS_ECUDA, std::string("panns_search_static: cudaGetSymbolAddress: ") +
                                         cudaGetErrorString(e));
        g_static_addr[device] = ptr;
    }
    *out = static_cast<unsigned char *>(g_static_addr[device]);
    return PANNS_OK;
}

}  // namespace

extern "C" int panns_search_static(panns_index *h, const panns_search_params *p, const float *d_queries,
                                   uint32_t nq, uint32_t *d_out_ids, void *stream) {
    if (!h || !p) return fail(PANNS_EINVAL, "panns_search_static: NULL argument");
    if (!h->ready)
        return fail(PANNS_ESTATE, "panns_search_static: the index is not laid out on the GPU yet; "
                                  "run one panns_search or panns_search_host first");
    if (p->mode != PANNS_MODE_NSG_SEQ && p->mode != PANNS_MODE_TOP_M &&
        !(p->mode == PANNS_MODE_PSS_V5 && p->T == 1))
        return fail(PANNS_EINVAL, "panns_search_static: only NSG_SEQ, TOP_M and PSS_V5 with T = 1");
    if (p->distance > PANNS_DIST_L2) return fail(PANNS_EINVAL, "panns_search_static: unknown distance");
    if (p->L == 0 || p->L > h->n) return fail(PANNS_EINVAL, "panns_search_static: need 0 < L <= N");
    if (p->K == 0 || p->K > p->L) return fail(PANNS_EINVAL, "panns_search_static: need 0 < K <= L");
    if (p->L > kStaticMaxL)
        return fail(PANNS_EINVAL, "panns_search_static: L = " + std::to_string(p->L) +
                                      " exceeds the fixed scratch limit of " + std::to_string(kStaticMaxL));
    if (p->mode == PANNS_MODE_TOP_M && (p->M == 0 || p->M > (uint32_t) kMaxM))
        return fail(PANNS_EINVAL, "panns_search_static: TOP_M needs 1 <= M <= 64");
    if (p->warps_per_block > 8 || p->flags || p->storage != PANNS_STORE_FP32 || p->L_query)
        return fail(PANNS_EINVAL, "panns_search_static: bad params (float32 storage, no flags, no L_query)");
    if (p->warps_per_query > 1 || p->blocks_per_sm)
        return fail(PANNS_EINVAL, "panns_search_static: runs one warp per query with as many blocks per SM "
                                  "as fit (warps_per_query <= 1, blocks_per_sm = 0)");
    if (nq == 0) return PANNS_OK;
    if (!d_queries || !d_out_ids) return fail(PANNS_EINVAL, "panns_search_static: NULL device buffer");
    cudaStream_t st = stream ? (cudaStream_t) stream : h->stream;
    CU(cudaSetDevice(h->device));
    unsigned char *base = nullptr;
    int rc = static_scratch_address(h->device, &base);
    if (rc) return rc;

    // Carve the fixed array: header | init ids | chain-major queries | cleared-word lists | bitsets.
    const uint32_t vis_words = (h->n + 31) / 32;
    const size_t off_init = kStaticHeader;
    const size_t off_q = off_init + (size_t) kStaticMaxL * 4;
    const size_t q_bytes = ((size_t) nq * h->dpad * 4 + 255) & ~(size_t) 255;
    const size_t off_slots = off_q + q_bytes;
    const size_t per_slot = (size_t) kStaticDirtyCap * 4 + (size_t) vis_words * 4;
    if (off_slots + per_slot > kStaticScratchBytes)
        return fail(PANNS_EINVAL, "panns_search_static: N = " + std::to_string(h->n) + " with nq = " +
                                      std::to_string(nq) + " does not fit the fixed " +
                                      std::to_string(kStaticScratchBytes >> 20) + " MiB scratch");
    const uint32_t fit_slots = (uint32_t) ((kStaticScratchBytes - off_slots) / per_slot);

    const int CL = (int) (h->dpad / 32);
    const uint32_t kind = p->distance == PANNS_DIST_L2 ? KIND_L2 : KIND_IP;
    const void *kern = search_kernel_ptr(kind, ORDER_PANNS, CL);
    if (!kern) return fail(PANNS_EINVAL, "panns_search_static: unsupported dimension");
    const uint32_t M = p->mode == PANNS_MODE_TOP_M ? p->M : 1u;
    const uint32_t qcap = ((p->L + 31) / 32) * 32;
    const uint32_t wpb = p->warps_per_block ? p->warps_per_block : 4u;
    const size_t smem = (size_t) wpb * warp_smem_bytes(qcap);
    {
        cudaFuncAttributes fa;
        CU(cudaFuncGetAttributes(&fa, kern));
        if ((int) (wpb * 32) > fa.maxThreadsPerBlock)
            return fail(PANNS_EINVAL, "search: warps_per_block must be <= " + std::to_string(fa.maxThreadsPerBlock / 32) +
                                          " for this kernel");
    }
    CU(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    CU(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, -1));
    int per_sm = 0;
    CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int) wpb * 32, smem));
    if (per_sm < 1) return fail(PANNS_EINVAL, "panns_search_static: L too large for shared memory");
    uint32_t blocks = std::min((uint32_t) per_sm * (uint32_t) h->num_sms, (nq + wpb - 1) / wpb);
    blocks = std::min(blocks, fit_slots / wpb);
    if (blocks == 0)
        return fail(PANNS_EINVAL, "panns_search_static: N = " + std::to_string(h->n) +
                                      " leaves room for fewer than one block of warps in the fixed scratch");
    const uint32_t slots = blocks * wpb;

    // Init ids: the PANNS list (fill_init_ids, shared with
    // panns_prepare_init_ids), as device ids, built in a stack buffer.
    uint32_t init[kStaticMaxL];
    const uint32_t end = p->L;
    fill_init_ids(h, end, init);
    for (uint32_t i = 0; i < end; ++i) init[i] = h->inv[init[i]];

    uint32_t *counter = reinterpret_cast<uint32_t *>(base);
    uint32_t *err_word = counter + 1;
    uint32_t *d_init = reinterpret_cast<uint32_t *>(base + off_init);
    float *d_qcm = reinterpret_cast<float *>(base + off_q);
    uint32_t *d_dirty = reinterpret_cast<uint32_t *>(base + off_slots);
    uint32_t *d_vis = d_dirty + (size_t) slots * kStaticDirtyCap;
    CU(cudaMemsetAsync(base, 0, kStaticHeader, st));
    CU(cudaMemsetAsync(d_vis, 0, (size_t) slots * vis_words * 4, st));
    CU(cudaMemcpyAsync(d_init, init, (size_t) end * 4, cudaMemcpyHostToDevice, st));
    {
        const uint64_t total = (uint64_t) nq * h->dpad;
        const int pb = (int) std::min<uint64_t>((total + 255) / 256, (uint64_t) h->num_sms * 32);
        permute_rows_kernel<<<std::max(pb, 1), 256, 0, st>>>(d_queries, d_qcm, nq, (int) h->d,
                                                             (int) h->dpad, nullptr);
        CU(cudaGetLastError());
    }
    SearchArgs a;
    memset(&a, 0, sizeof(a));
    a.vec = reinterpret_cast<const float4 *>(h->vec.p);
    a.norms = h->norms.p;
    a.head = h->head.p;
    a.ovf_off = h->ovf_off.p;
    a.ovf = h->ovf.p;
    a.orig = h->orig.p;
    a.vec_lo = nullptr;
    a.norms_lo = nullptr;
    a.scales = nullptr;
    a.d = h->d;
    a.n = h->n;
    a.queries = reinterpret_cast<const float4 *>(d_qcm);
    a.nq = nq;
    a.init_ids = d_init;
    a.init_stride = 0;
    a.K = p->K;
    a.L = p->L;
    a.M = M;
    a.out_ids = d_out_ids;
    a.out_stats = nullptr;
    a.visited = d_vis;
    a.vis_words = vis_words;
    a.dirty = d_dirty;
    a.dirty_cap = kStaticDirtyCap;
    a.counter = counter;
    a.error = err_word;
    a.queue_cap = qcap;
    void *args[] = {&a};
    CU(cudaLaunchKernel(kern, dim3(blocks), dim3(wpb * 32), args, smem, st));
    uint32_t err = 0;
    CU(cudaMemcpyAsync(&err, err_word, 4, cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    if (err & ERR_BAD_ID) return fail(PANNS_EDEVICE, "panns_search_static: a neighbour id >= N");
    if (err & ERR_BAD_INIT) return fail(PANNS_EDEVICE, "panns_search_static: init id >= N");
    return PANNS_OK;
}

// ---- learned entry / L budget -----------------------------------------------

extern "C" int panns_kmeans(panns_index *h, uint32_t k, uint32_t iters, uint32_t seed, uint32_t *rep_ids,
                            uint32_t *assign, float *centroids) {
    if (!h) return fail(PANNS_EINVAL, "panns_kmeans: NULL handle");
    if (!h->n || !h->base_raw.p) return fail(PANNS_ESTATE, "panns_kmeans: no base vectors loaded");
    CU(cudaSetDevice(h->device));
    DevBuf<float> cent;
    DevBuf<uint32_t> as, rep;
    CU(cent.ensure((size_t) k * h->d));
    CU(as.ensure(h->n));
    CU(rep.ensure(k));
    int rc = panns::kmeans_run(h->base_raw.p, h->n, h->d, k, iters, seed, cent.p, as.p, rep.p, h->stream);
    if (rc) return rc;
    if (rep_ids) CU(cudaMemcpyAsync(rep_ids, rep.p, k * 4ull, cudaMemcpyDeviceToHost, h->stream));
    if (assign) CU(cudaMemcpyAsync(assign, as.p, h->n * 4ull, cudaMemcpyDeviceToHost, h->stream));
    if (centroids)
        CU(cudaMemcpyAsync(centroids, cent.p, (size_t) k * h->d * 4, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    return PANNS_OK;
}

extern "C" int panns_set_learned(panns_index *h, const float *params, uint32_t R, const uint32_t *rep_ids,
                                 const panns_learned_params *lp) {
    if (!h || !params || !rep_ids || !lp) return fail(PANNS_EINVAL, "panns_set_learned: NULL argument");
    int rc = finalize(h);
    if (rc) return rc;
    if (R == 0 || R > (uint32_t) kMlpMaxR || R % kMlpH)
        return fail(PANNS_EINVAL, "panns_set_learned: need R a multiple of 256, R <= 4096");
    if (lp->E > (uint32_t) kMlpMaxE) return fail(PANNS_EINVAL, "panns_set_learned: need E <= 64");
    if (!(lp->min_conf >= 0.f && lp->min_conf <= 1.f))
        return fail(PANNS_EINVAL, "panns_set_learned: need 0 <= min_conf <= 1");
    if (lp->use_L && !(lp->L_scale > 0.f)) return fail(PANNS_EINVAL, "panns_set_learned: need L_scale > 0");
    std::vector<uint32_t> rep(R);
    for (uint32_t i = 0; i < R; ++i) {
        if (rep_ids[i] >= h->n) return fail(PANNS_EINVAL, "panns_set_learned: representative id >= N");
        rep[i] = h->inv[rep_ids[i]];
    }
    CU(cudaSetDevice(h->device));
    // Searches still in flight (on any stream) read the network being replaced.
    CU(cudaDeviceSynchronize());
    const uint64_t P = panns_mlp_param_count(h->d, R);
    DevBuf<float> dp;
    CU(dp.ensure(P));
    // Every copy goes on the handle's stream, which the packing kernel and the
    // searches use: a plain cudaMemcpy from pageable memory may return before
    // its DMA lands, and that stream (non-blocking) is not ordered after it.
    CU(cudaMemcpyAsync(dp.p, params, P * 4, cudaMemcpyHostToDevice, h->stream));
    CU(h->mlp_w.ensure((size_t) kMlpH * (h->d + kMlpH + R)));
    CU(h->mlp_f.ensure(3u * kMlpH + R + 1));
    CU(h->mlp_rep.ensure(R));
    rc = panns::mlp_pack_inference(dp.p, h->d, R, h->mlp_w.p, h->mlp_f.p, h->stream);
    if (rc) return rc;
    CU(cudaMemcpyAsync(h->mlp_rep.p, rep.data(), R * 4ull, cudaMemcpyHostToDevice, h->stream));
    float bl = 0.f;
    CU(cudaMemcpyAsync(&bl, h->mlp_f.p + 3u * kMlpH + R, 4, cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    MlpDev m{};
    const __nv_bfloat16 *wb = reinterpret_cast<const __nv_bfloat16 *>(h->mlp_w.p);
    m.w1 = wb;
    m.w2 = wb + (size_t) h->d * kMlpH;
    m.w3 = wb + (size_t) (h->d + kMlpH) * kMlpH;
    m.b1 = h->mlp_f.p;
    m.b2 = h->mlp_f.p + kMlpH;
    m.b3 = h->mlp_f.p + 2 * kMlpH;
    m.wl = h->mlp_f.p + 2 * kMlpH + R;
    m.bl = bl;
    m.rep = h->mlp_rep.p;
    m.d = h->d;
    m.R = R;
    m.E = lp->E;
    m.L_init = lp->L_init;
    m.L_min = lp->L_min;
    m.use_entry = lp->E > 0;
    m.use_L = lp->use_L;
    m.min_conf = lp->min_conf;
    m.L_scale = lp->L_scale;
    m.L_exp = lp->L_exp;
    if (h->mlp.R != R) h->mlp_chunk = 0;  // the inference scratch is re-sized at the next launch
    h->mlp = m;
    h->has_mlp = true;
    return PANNS_OK;
}

extern "C" int panns_learned_record(panns_index *h, uint32_t nq, uint32_t *out) {
    if (!h || (nq && !out)) return fail(PANNS_EINVAL, "panns_learned_record: NULL argument");
    if (nq > h->mlp_last_nq) return fail(PANNS_EINVAL, "panns_learned_record: nq exceeds the last learned call");
    if (nq == 0) return PANNS_OK;
    CU(cudaSetDevice(h->device));
    CU(cudaStreamSynchronize(h->stream));
    CU(cudaMemcpy(out, h->mlp_record.p, (size_t) nq * kMlpRecWords * 4, cudaMemcpyDeviceToHost));
    for (uint32_t q = 0; q < nq; ++q) {  // entries as original ids
        uint32_t *r = out + (size_t) q * kMlpRecWords;
        const uint32_t E = std::min<uint32_t>(r[1], kMlpMaxE);
        for (uint32_t i = 0; i < E; ++i) r[2 + i] = r[2 + i] < h->n ? h->perm[r[2 + i]] : r[2 + i];
    }
    return PANNS_OK;
}

int32_t panns::glibc_rand_next(int32_t *st) { return rand_next(st); }

#ifdef PANNS_DEBUG_VISITED
// Diagnostic builds only: the number of non-zero words left in the handle's
// visited bitsets (zero between calls when every query cleared its bits).
extern "C" int panns_debug_visited_nonzero(panns_index *h, uint64_t *count) {
    if (!h || !count) return fail(PANNS_EINVAL, "NULL argument");
    CU(cudaSetDevice(h->device));
    CU(cudaDeviceSynchronize());
    std::vector<uint32_t> v((size_t) h->vis_slots * h->vis_words);
    if (!v.empty()) CU(cudaMemcpy(v.data(), h->visited.p, v.size() * 4, cudaMemcpyDeviceToHost));
    uint64_t c = 0;
    for (uint32_t w : v) c += w != 0;
    *count = c;
    return PANNS_OK;
}
#endif
