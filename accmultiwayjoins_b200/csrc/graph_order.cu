// Degree ordering of an oriented edge relation.
//
// When every edge (u, v) of a self-joined relation has 0 <= u < v, the
// triangles (and 4-cliques) of the join in attribute order are exactly the
// increasing triples (quadruples) of the undirected graph, each once.  Any
// acyclic orientation lists each of them once too, so an operator may join
// the copy oriented from the lower to the higher (degree, id) and report
// every tuple in increasing order: the same bag, the same checksum.  Hub
// vertices then keep short child lists.  Used by ALFTJ (triangle, 4-clique)
// and by AMHJ TRI / FOUR.
#include "amj_ops.cuh"

#include <algorithm>

namespace amj {

__global__ void orient_check_kernel(const int32_t *__restrict__ s, const int32_t *__restrict__ d, uint64_t n,
                                    unsigned int *bad, int *maxv) {
    unsigned int b = 0;
    int m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t u = s[i], v = d[i];
        b |= (u < 0 || u >= v) ? 1u : 0u;
        m = v > m ? v : m;
    }
    b = __reduce_or_sync(AMJ_FULL_MASK, b);
    m = __reduce_max_sync(AMJ_FULL_MASK, m);
    if ((threadIdx.x & 31) == 0) {
        if (b) atomicOr(bad, 1u);
        atomicMax(maxv, m);
    }
}

__global__ void degree_kernel(const int32_t *__restrict__ s, const int32_t *__restrict__ d, uint64_t n,
                              unsigned int *deg) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        atomicAdd(&deg[s[i]], 1u);
        atomicAdd(&deg[d[i]], 1u);
    }
}

__global__ void reorient_kernel(const int32_t *__restrict__ s, const int32_t *__restrict__ d, uint64_t n,
                                const unsigned int *__restrict__ deg, int32_t *__restrict__ ns,
                                int32_t *__restrict__ nd) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t u = s[i], v = d[i];
        const uint64_t ku = ((uint64_t)deg[u] << 32) | (uint32_t)u, kv = ((uint64_t)deg[v] << 32) | (uint32_t)v;
        ns[i] = ku < kv ? u : v;
        nd[i] = ku < kv ? v : u;
    }
}

int degree_ordered_copy(amj_ctx *ctx, const int32_t *c0, const int32_t *c1, uint64_t n, DBuf<int32_t> *ns,
                        DBuf<int32_t> *nd, bool *oriented) {
    *oriented = false;
    if (n == 0) return AMJ_OK;
    struct Probe {
        unsigned int bad;
        int maxv;
    };
    DBuf<Probe> pr;
    AMJ_TRY(pr.alloc(ctx, 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(pr.p, 0, sizeof(Probe), ctx->stream));
    const unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 16);
    note_launch(ctx);
    orient_check_kernel<<<g, 256, 0, ctx->stream>>>(c0, c1, n, &pr.p->bad, &pr.p->maxv);
    AMJ_CUDA_TRY(cudaGetLastError());
    Probe h;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h, pr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (h.bad) return AMJ_OK;
    // per-vertex arrays are sized by the largest id: sparse ids keep the
    // relation's own order instead
    if ((uint64_t)h.maxv + 1 > 4 * n + (1ull << 20)) return AMJ_OK;
    DBuf<unsigned int> deg;
    AMJ_TRY(deg.alloc(ctx, (uint64_t)h.maxv + 1));
    AMJ_TRY(ns->alloc(ctx, n));
    AMJ_TRY(nd->alloc(ctx, n));
    AMJ_CUDA_TRY(cudaMemsetAsync(deg.p, 0, ((uint64_t)h.maxv + 1) * sizeof(unsigned int), ctx->stream));
    note_launch(ctx);
    degree_kernel<<<g, 256, 0, ctx->stream>>>(c0, c1, n, deg.p);
    note_launch(ctx);
    reorient_kernel<<<g, 256, 0, ctx->stream>>>(c0, c1, n, deg.p, ns->p, nd->p);
    AMJ_CUDA_TRY(cudaGetLastError());
    *oriented = true;
    return AMJ_OK;
}

// degrees counted on every stride-th edge: an estimate that keeps the order
// of the hubs (the counts that matter for the orientation) at a fraction of
// the atomics; any total order gives the same join result
// The counts of ids below DEG_SMEM_IDS (where generators and real graphs put
// their hubs first: R-MAT's low ids) gather in shared memory per block and
// reach the global array once per block, so a hub's increments do not
// serialise on one global counter.
constexpr uint32_t DEG_SMEM_IDS = 8192;

__global__ void degree_sample_kernel(const int32_t *__restrict__ s, const int32_t *__restrict__ d, uint64_t n,
                                     uint32_t stride, uint64_t nv, unsigned int *deg) {
    __shared__ unsigned int h[DEG_SMEM_IDS];
    for (uint32_t i = threadIdx.x; i < DEG_SMEM_IDS; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const uint64_t m = (n + stride - 1) / stride;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t a = (uint32_t)s[i * stride], b = (uint32_t)d[i * stride];
        if (a < DEG_SMEM_IDS) atomicAdd(&h[a], 1u);
        else atomicAdd(&deg[a], 1u);
        if (b < DEG_SMEM_IDS) atomicAdd(&h[b], 1u);
        else atomicAdd(&deg[b], 1u);
    }
    __syncthreads();
    const uint32_t top = nv < DEG_SMEM_IDS ? (uint32_t)nv : DEG_SMEM_IDS;
    for (uint32_t i = threadIdx.x; i < top; i += blockDim.x)
        if (h[i]) atomicAdd(&deg[i], h[i]);
}

// the largest of nv degrees
__global__ void degree_max_kernel(const unsigned int *__restrict__ deg, uint64_t nv, unsigned int *out) {
    unsigned int m = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nv; i += (uint64_t)gridDim.x * blockDim.x)
        m = max(m, deg[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(AMJ_FULL_MASK, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// key (degree << idbits | id) of every vertex id in [0, nv)
__global__ void rank_keys_kernel(const unsigned int *__restrict__ deg, uint64_t nv, int idbits,
                                 uint64_t *__restrict__ keys) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nv; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = ((uint64_t)deg[i] << idbits) | i;
}

// rank[id] and inv[rank] from the sorted keys
__global__ void rank_scatter_kernel(const uint64_t *__restrict__ sorted, uint64_t nv, int idbits,
                                    int32_t *__restrict__ rank, int32_t *__restrict__ inv) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nv; i += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t id = (int32_t)(sorted[i] & ((1ull << idbits) - 1));
        inv[i] = id;
        rank[id] = (int32_t)i;
    }
}

__global__ void rank_edges_kernel(const int32_t *__restrict__ s, const int32_t *__restrict__ d, uint64_t n,
                                  const int32_t *__restrict__ rank, int32_t *__restrict__ ns, int32_t *__restrict__ nd) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const int32_t ru = rank[s[i]], rv = rank[d[i]];
        ns[i] = ru < rv ? ru : rv;
        nd[i] = ru < rv ? rv : ru;
    }
}

int degree_ranks(amj_ctx *ctx, const int32_t *c0, const int32_t *c1, uint64_t n, DBuf<int32_t> *rank,
                 DBuf<int32_t> *inv, uint64_t *nv, bool *oriented) {
    *oriented = false;
    *nv = 0;
    if (n == 0) return AMJ_OK;
    struct Probe {
        unsigned int bad;
        int maxv;
    };
    DBuf<Probe> pr;
    AMJ_TRY(pr.alloc(ctx, 1));
    AMJ_CUDA_TRY(cudaMemsetAsync(pr.p, 0, sizeof(Probe), ctx->stream));
    const unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 16);
    note_launch(ctx);
    orient_check_kernel<<<g, 256, 0, ctx->stream>>>(c0, c1, n, &pr.p->bad, &pr.p->maxv);
    AMJ_CUDA_TRY(cudaGetLastError());
    Probe h;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&h, pr.p, sizeof(h), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (h.bad) return AMJ_OK;
    const uint64_t V = (uint64_t)h.maxv + 1;
    // per-vertex arrays are sized by the largest id: sparse ids keep the
    // relation's own order instead
    if (V > 4 * n + (1ull << 20)) return AMJ_OK;
    DBuf<unsigned int> deg;
    AMJ_TRY(deg.alloc(ctx, V));
    AMJ_CUDA_TRY(cudaMemsetAsync(deg.p, 0, V * sizeof(unsigned int), ctx->stream));
    // relations of 2^20 edges or more rank by degrees counted on every 4th edge
    const uint32_t stride = n >= (1ull << 20) ? 4u : 1u;
    note_launch(ctx);
    degree_sample_kernel<<<(unsigned)std::min<uint64_t>(g, (uint64_t)ctx->num_sms * 4), 256, 0, ctx->stream>>>(
        c0, c1, n, stride, V, deg.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    DBuf<uint64_t> ka, kb;
    AMJ_TRY(ka.alloc(ctx, V));
    AMJ_TRY(kb.alloc(ctx, V));
    const unsigned gv = (unsigned)std::min<uint64_t>((V + 255) / 256, (uint64_t)ctx->num_sms * 16);
    // the largest degree sets the key width: keys of idbits + degbits bits
    AMJ_CUDA_TRY(cudaMemsetAsync(&pr.p->bad, 0, sizeof(unsigned int), ctx->stream));
    note_launch(ctx);
    degree_max_kernel<<<gv, 256, 0, ctx->stream>>>(deg.p, V, &pr.p->bad);
    AMJ_CUDA_TRY(cudaGetLastError());
    unsigned int maxdeg = 0;
    AMJ_CUDA_TRY(cudaMemcpyAsync(&maxdeg, &pr.p->bad, sizeof(maxdeg), cudaMemcpyDeviceToHost, ctx->stream));
    AMJ_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    int idbits = 1, degbits = 1;
    while (idbits < 31 && (V - 1) >> idbits) idbits++;
    while (degbits < 32 && (uint64_t)maxdeg >> degbits) degbits++;
    if (idbits + degbits > 64) return fail(AMJ_EUNSUPPORTED, "degree ranks: relation too large");
    note_launch(ctx);
    rank_keys_kernel<<<gv, 256, 0, ctx->stream>>>(deg.p, V, idbits, ka.p);
    AMJ_CUDA_TRY(cudaGetLastError());
    // the keys start in id order and the sort is stable: sorting the degree
    // bits alone leaves them in (degree, id) order
    uint64_t *sorted = nullptr;
    AMJ_TRY(radix_sort_u64(ctx, ka.p, kb.p, V, SK_IDENT, idbits, idbits + degbits, &sorted));
    AMJ_TRY(rank->alloc(ctx, V));
    AMJ_TRY(inv->alloc(ctx, V));
    note_launch(ctx);
    rank_scatter_kernel<<<gv, 256, 0, ctx->stream>>>(sorted, V, idbits, rank->p, inv->p);
    AMJ_CUDA_TRY(cudaGetLastError());
    *nv = V;
    *oriented = true;
    return AMJ_OK;
}

int degree_ranked_copy(amj_ctx *ctx, const int32_t *c0, const int32_t *c1, uint64_t n, DBuf<int32_t> *ns,
                       DBuf<int32_t> *nd, DBuf<int32_t> *inv, uint64_t *nv, bool *oriented) {
    DBuf<int32_t> rank;
    AMJ_TRY(degree_ranks(ctx, c0, c1, n, &rank, inv, nv, oriented));
    if (!*oriented) return AMJ_OK;
    AMJ_TRY(ns->alloc(ctx, n));
    AMJ_TRY(nd->alloc(ctx, n));
    const unsigned g = (unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)ctx->num_sms * 16);
    note_launch(ctx);
    rank_edges_kernel<<<g, 256, 0, ctx->stream>>>(c0, c1, n, rank.p, ns->p, nd->p);
    AMJ_CUDA_TRY(cudaGetLastError());
    return AMJ_OK;
}

}  // namespace amj
