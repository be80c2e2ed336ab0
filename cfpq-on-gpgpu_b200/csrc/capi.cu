// C ABI of libcfpq_b200.so (declared in include/cfpq_b200.h).
//
// Host runtime: context (device, stream, scratch buffers, delta-matrix pool,
// cached CUDA graph), matrices, product entry point and the two closure
// drivers:
//   ENGINE   -- semi-naive iterations resident on the device.  Iteration t
//               runs, for every rule C -> A B, the product terms
//               dA_{t-1} * B and A * dB_{t-1} (d = bits added in the previous
//               iteration; in the first iteration dA = A and only the first
//               term runs).  New bits of C go to C and to dC_t.  The loop ends
//               after an iteration without new bits.  Every bit of the least
//               fixpoint is produced because each pair (A bit, B bit) meets in
//               the iteration after the later of the two appeared.  Iterations
//               are plan -> product -> advance+end kernels, either
//               launched from a host loop that checks the flag every few
//               iterations or captured once as the body of a CUDA-graph while
//               node whose condition the last block of the advance+end kernel
//               sets on the device.
//   WORKLIST -- the reference loop (cfpq-cpp/Grammar.h:58-69): one add_mul at
//               a time with the changed flag read back after each product.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <string>
#include <unordered_map>
#include <vector>

#include "ctx.h"

static void free_plan_cache(cfpq_ctx *ctx);

// ---------------------------------------------------------------------------
// errors

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

// ---------------------------------------------------------------------------
// helpers

static inline uint32_t tiles_for(uint32_t n) { return (n + 63) / 64; }

// Iterations of a persistent closure whose phase timestamps are kept.
constexpr uint32_t kPhaseLogIters = 4096;
// Iterations of a closure whose selection rows are kept.
constexpr uint32_t kSelLogIters = 128;

// Upper bound of the work items one product term can emit per iteration:
// tile-rows x column blocks x chunks per block (tensor-core items: fewer).
static inline size_t item_capacity(uint32_t T, int tpb) {
    return (size_t)T * ((T + tpb - 1) / tpb) * kMaxChunksPerBlock;
}

static int alloc_devmat(uint32_t n, DevMat *d) {
    memset(d, 0, sizeof(*d));
    d->n = n;
    d->T = tiles_for(n);
    d->ow = (d->T + 31) / 32;
    if (d->T == 0) return CFPQ_OK;
    const size_t bits_bytes = (size_t)d->T * d->T * 512;
    const size_t occ_bytes = (size_t)d->T * d->ow * 4;
    cudaError_t e = cudaMalloc(&d->bits, bits_bytes);
    if (e != cudaSuccess)
        return set_error(CFPQ_ERR_OOM, "cannot allocate %zu bytes for a %u x %u matrix: %s", bits_bytes, n, n,
                         cudaGetErrorString(e));
    e = cudaMalloc(&d->occ, occ_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&d->nnz, (size_t)d->T * d->T * 4);
    if (e != cudaSuccess) {
        cudaFree(d->bits);
        if (d->occ) cudaFree(d->occ);
        d->bits = nullptr;
        d->occ = nullptr;
        d->nnz = nullptr;
        return set_error(CFPQ_ERR_OOM, "cannot allocate tile statistics: %s", cudaGetErrorString(e));
    }
    return CFPQ_OK;
}

static void free_devmat(DevMat *d) {
    if (d->bits) cudaFree(d->bits);
    if (d->occ) cudaFree(d->occ);
    if (d->nnz) cudaFree(d->nnz);
    d->bits = nullptr;
    d->occ = nullptr;
    d->nnz = nullptr;
}

static int use_device(cfpq_ctx *ctx) {
    if (!ctx) return set_error(CFPQ_ERR_INVALID, "null context");
    CUDA_TRY(cudaSetDevice(ctx->device));
    return CFPQ_OK;
}

// Take a zeroed matrix of size n from the pool (or allocate one).
static int pool_take(cfpq_ctx *ctx, uint32_t n, cfpq_matrix **out) {
    for (size_t i = 0; i < ctx->pool.size(); ++i) {
        if (ctx->pool[i]->d.n == n) {
            *out = ctx->pool[i];
            ctx->pool.erase(ctx->pool.begin() + i);
            return CFPQ_OK;
        }
    }
    cfpq_matrix *m = new cfpq_matrix();
    m->ctx = ctx;
    int rc = alloc_devmat(n, &m->d);
    if (rc != CFPQ_OK) {
        delete m;
        return rc;
    }
    cudaError_t e = launch_clear_matrix(m->d, ctx->stream);
    if (e != cudaSuccess) {
        free_devmat(&m->d);
        delete m;
        return set_error(CFPQ_ERR_CUDA, "clear: %s", cudaGetErrorString(e));
    }
    *out = m;
    return CFPQ_OK;
}

// Return a matrix to the pool; `dirty` matrices are cleared first.
static int pool_give(cfpq_ctx *ctx, cfpq_matrix *m, bool dirty) {
    if (dirty) CUDA_TRY(launch_clear_matrix(m->d, ctx->stream));
    ctx->pool.push_back(m);
    return CFPQ_OK;
}

// Hash power tables for vertex ids 0..n-1 stored at internal index perm[v]
// (identity when perm is null): pow11[perm[c]] = 11^(n-1-c),
// pow13[perm[r]] = 13^(n-1-r) modulo 1e9+7 (cfpq-cpp/Grammar.cpp:12-14),
// and the nibble tables of pow11 the hash kernel reads (built on stream s).
static int make_pow_tables(uint32_t n, const uint32_t *perm, PowTables *t, cudaStream_t s) {
    const uint32_t np = tiles_for(n) * 64;
    std::vector<uint32_t> p11(np ? np : 1, 0), p13(np ? np : 1, 0);
    const uint64_t mod = 1000000007ULL;
    uint64_t a = 1, b = 1;
    for (int64_t c = (int64_t)n - 1; c >= 0; --c) {
        const uint32_t at = perm ? perm[c] : (uint32_t)c;
        p11[at] = (uint32_t)a;
        p13[at] = (uint32_t)b;
        a = a * 11 % mod;
        b = b * 13 % mod;
    }
    CUDA_TRY(cudaMalloc(&t->d_pow11, p11.size() * 4));
    CUDA_TRY(cudaMalloc(&t->d_pow13, p13.size() * 4));
    CUDA_TRY(cudaMemcpy(t->d_pow11, p11.data(), p11.size() * 4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(t->d_pow13, p13.data(), p13.size() * 4, cudaMemcpyHostToDevice));
    const uint32_t T = tiles_for(n);
    CUDA_TRY(cudaMalloc(&t->d_nib11, (size_t)(T ? T : 1) * 256 * 4));
    if (T) CUDA_TRY(launch_pow_nibbles(t->d_pow11, T, t->d_nib11, s));
    return CFPQ_OK;
}

static int get_pow_tables(cfpq_ctx *ctx, const cfpq_matrix *m, PowTables *out) {
    if (m->order) {
        *out = m->order->pow;
        return CFPQ_OK;
    }
    const uint32_t n = m->d.n;
    auto it = ctx->pow.find(n);
    if (it != ctx->pow.end()) {
        *out = it->second;
        return CFPQ_OK;
    }
    PowTables t;
    TRY(make_pow_tables(n, nullptr, &t, ctx->stream));
    ctx->pow[n] = t;
    *out = t;
    return CFPQ_OK;
}

extern "C" int cfpq_order_create(cfpq_ctx *ctx, uint32_t n, const uint32_t *perm, cfpq_order **out) {
    TRY(use_device(ctx));
    if (!out || (n && !perm)) return set_error(CFPQ_ERR_INVALID, "null argument");
    std::vector<char> seen(n, 0);
    for (uint32_t v = 0; v < n; ++v) {
        if (perm[v] >= n || seen[perm[v]]) return set_error(CFPQ_ERR_INVALID, "perm is not a permutation of 0..%u", n - 1);
        seen[perm[v]] = 1;
    }
    cfpq_order *o = new cfpq_order();
    o->n = n;
    if (n) {
        cudaError_t e = cudaMalloc(&o->d_perm, (size_t)n * 4);
        if (e == cudaSuccess) e = cudaMemcpy(o->d_perm, perm, (size_t)n * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            if (o->d_perm) cudaFree(o->d_perm);
            delete o;
            return set_error(CFPQ_ERR_CUDA, "order upload: %s", cudaGetErrorString(e));
        }
    }
    int rc = make_pow_tables(n, n ? perm : nullptr, &o->pow, ctx->stream);
    if (rc != CFPQ_OK) {
        if (o->d_perm) cudaFree(o->d_perm);
        delete o;
        return rc;
    }
    *out = o;
    return CFPQ_OK;
}

extern "C" int cfpq_order_destroy(cfpq_ctx *ctx, cfpq_order *order) {
    if (!order) return CFPQ_OK;
    TRY(use_device(ctx));
    cudaStreamSynchronize(ctx->stream);
    if (order->d_perm) cudaFree(order->d_perm);
    if (order->pow.d_pow11) cudaFree(order->pow.d_pow11);
    if (order->pow.d_pow13) cudaFree(order->pow.d_pow13);
    if (order->pow.d_nib11) cudaFree(order->pow.d_nib11);
    delete order;
    return CFPQ_OK;
}

static int sync_and_check(cfpq_ctx *ctx) {
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return CFPQ_OK;
}

// ---------------------------------------------------------------------------
// context

extern "C" int cfpq_abi_version(void) { return CFPQ_B200_ABI_VERSION; }

extern "C" const char *cfpq_last_error(void) { return g_last_error.c_str(); }

extern "C" int cfpq_ctx_create(int device, cfpq_ctx **out) {
    if (!out) return set_error(CFPQ_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    CUDA_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return set_error(CFPQ_ERR_INVALID, "device %d out of range (%d devices)", device, ndev);
    CUDA_TRY(cudaSetDevice(device));
    cfpq_ctx *c = new cfpq_ctx();
    c->device = device;
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        delete c;
        return set_error(CFPQ_ERR_UNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a", device,
                         prop.major, prop.minor);
    }
    c->num_sms = prop.multiProcessorCount;
    CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&c->ev0));
    CUDA_TRY(cudaEventCreate(&c->ev1));
    for (auto &e : c->kev) CUDA_TRY(cudaEventCreate(&e));
    CUDA_TRY(cudaMalloc(&c->d_st, sizeof(IterState)));
    CUDA_TRY(cudaMalloc(&c->d_flag, 64));
    CUDA_TRY(cudaMalloc(&c->d_bad, 64));
    CUDA_TRY(cudaMallocHost(&c->h_st, sizeof(IterState)));
    CUDA_TRY(cudaMallocHost(&c->h_flag, 64));
    // the persistent kernel writes its final state straight into these
    // (device views of the pinned blocks; without them it is copied back)
    if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&c->h_st_dev), c->h_st, 0) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&c->h_flag_dev), c->h_flag, 0) != cudaSuccess) {
        c->h_st_dev = nullptr;
        c->h_flag_dev = nullptr;
        (void)cudaGetLastError();
    }
    c->lop3_grid = c->num_sms * product_tiled_blocks_per_sm(0);
    c->m4r_grid = c->num_sms * product_tiled_blocks_per_sm(1);
    // The tensor-core kernel allocates all 512 TMEM columns of its SM, so it
    // must run one CTA per SM; it is only enabled when that is guaranteed.
    c->tc_grid = product_tc_blocks_per_sm() == 1 ? c->num_sms : 0;
    int coop = 0;
    cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device);
    for (int m = 0; m < 2; ++m) c->persist_grid[m] = coop ? persistent_blocks_per_sm(m) * c->num_sms : 0;
    selector_defaults(&c->sel);
    if (!c->tc_grid) c->sel.allowed &= ~(1u << CFPQ_VARIANT_TC);
    *out = c;
    return CFPQ_OK;
}

extern "C" int cfpq_ctx_destroy(cfpq_ctx *ctx) {
    if (!ctx) return CFPQ_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    ctx->gcache.release();
    free_plan_cache(ctx);
    for (auto *m : ctx->pool) {
        free_devmat(&m->d);
        delete m;
    }
    for (auto &kv : ctx->pow) {
        cudaFree(kv.second.d_pow11);
        cudaFree(kv.second.d_pow13);
        cudaFree(kv.second.d_nib11);
    }
    for (DevBuf *b : {&ctx->stage, &ctx->items, &ctx->prods, &ctx->slots, &ctx->qtrack, &ctx->prod_seen,
                      &ctx->mats_desc, &ctx->edge_buf, &ctx->phase_log, &ctx->clear_desc, &ctx->diag_desc,
                      &ctx->d_sel, &ctx->cnts, &ctx->choice, &ctx->tc_ok, &ctx->sel_log, &ctx->tc_rows, &ctx->mlp_w, &ctx->mlp_x,
                      &ctx->mlp_y, &ctx->mlp_m, &ctx->mlp_grad, &ctx->mlp_m1, &ctx->mlp_v2, &ctx->mlp_loss,
                      &ctx->mlp_out, &ctx->qranges, &ctx->item_trace, &ctx->nt_cells, &ctx->nt_mats,
                      &ctx->nt_rules, &ctx->nt_ctr})
        b->release();
    cudaFree(ctx->d_st);
    cudaFree(ctx->d_flag);
    cudaFree(ctx->d_bad);
    if (ctx->d_hash) cudaFree(ctx->d_hash);
    if (ctx->d_hash_part) cudaFree(ctx->d_hash_part);
    if (ctx->d_hash_ticket) cudaFree(ctx->d_hash_ticket);
    cudaFreeHost(ctx->h_st);
    cudaFreeHost(ctx->h_flag);
    if (ctx->h_hash) cudaFreeHost(ctx->h_hash);
    if (ctx->h_small) cudaFreeHost(ctx->h_small);
    if (ctx->h_query) cudaFreeHost(ctx->h_query);
    cudaEventDestroy(ctx->ev0);
    cudaEventDestroy(ctx->ev1);
    for (auto &e : ctx->kev) cudaEventDestroy(e);
    for (auto &e : ctx->tev) cudaEventDestroy(e);
    cudaStreamDestroy(ctx->stream);
    delete ctx;
    return CFPQ_OK;
}

extern "C" int cfpq_ctx_synchronize(cfpq_ctx *ctx) {
    TRY(use_device(ctx));
    return sync_and_check(ctx);
}

extern "C" int cfpq_ctx_num_sms(const cfpq_ctx *ctx) { return ctx ? ctx->num_sms : 0; }

// ---------------------------------------------------------------------------
// matrices

extern "C" int cfpq_matrix_create(cfpq_ctx *ctx, uint32_t n, cfpq_matrix **out) {
    return cfpq_matrix_create_ordered(ctx, n, nullptr, out);
}

extern "C" int cfpq_matrix_create_ordered(cfpq_ctx *ctx, uint32_t n, cfpq_order *order, cfpq_matrix **out) {
    TRY(use_device(ctx));
    if (!out) return set_error(CFPQ_ERR_INVALID, "null output pointer");
    if (order && order->n != n) return set_error(CFPQ_ERR_INVALID, "order is for %u vertices, matrix has %u", order->n, n);
    if (tiles_for(n) > (uint32_t)product_lop3_max_tiles())
        return set_error(CFPQ_ERR_UNSUPPORTED, "n = %u exceeds the supported maximum %d", n,
                         product_lop3_max_tiles() * 64);
    cfpq_matrix *m = new cfpq_matrix();
    m->ctx = ctx;
    m->order = order;
    int rc = alloc_devmat(n, &m->d);
    m->d.perm = order ? order->d_perm : nullptr;
    if (rc != CFPQ_OK) {
        delete m;
        return rc;
    }
    cudaError_t e = launch_clear_matrix(m->d, ctx->stream);
    if (e != cudaSuccess) {
        free_devmat(&m->d);
        delete m;
        return set_error(CFPQ_ERR_CUDA, "clear: %s", cudaGetErrorString(e));
    }
    *out = m;
    return CFPQ_OK;
}

extern "C" int cfpq_matrix_destroy(cfpq_ctx *ctx, cfpq_matrix *m) {
    if (!m) return CFPQ_OK;
    TRY(use_device(ctx));
    cudaStreamSynchronize(ctx->stream);
    free_devmat(&m->d);
    delete m;
    return CFPQ_OK;
}

extern "C" uint32_t cfpq_matrix_size(const cfpq_matrix *m) { return m ? m->d.n : 0; }

static int check_bad(cfpq_ctx *ctx, const char *what) {
    uint32_t bad = 0;
    CUDA_TRY(cudaMemcpyAsync(ctx->h_flag, ctx->d_bad, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    bad = ctx->h_flag[0];
    if (bad) return set_error(CFPQ_ERR_INVALID, "%s: %u coordinates out of range", what, bad);
    return CFPQ_OK;
}

extern "C" int cfpq_matrix_set_bits(cfpq_ctx *ctx, cfpq_matrix *m, const uint32_t *rows, const uint32_t *cols,
                                    size_t count) {
    TRY(use_device(ctx));
    if (!m || (count && (!rows || !cols))) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (count == 0) return CFPQ_OK;
    TRY(ctx->stage.ensure(count * 8));
    uint32_t *dr = ctx->stage.as<uint32_t>(), *dc = dr + count;
    CUDA_TRY(cudaMemcpyAsync(dr, rows, count * 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(dc, cols, count * 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemsetAsync(ctx->d_bad, 0, 4, ctx->stream));
    CUDA_TRY(launch_set_bits(m->d, dr, dc, count, ctx->d_bad, ctx->stream));
    return check_bad(ctx, "cfpq_matrix_set_bits");
}

extern "C" int cfpq_matrix_set_bits_device(cfpq_ctx *ctx, cfpq_matrix *m, const uint32_t *d_rows,
                                           const uint32_t *d_cols, size_t count) {
    TRY(use_device(ctx));
    if (!m || (count && (!d_rows || !d_cols))) return set_error(CFPQ_ERR_INVALID, "null argument");
    CUDA_TRY(cudaMemsetAsync(ctx->d_bad, 0, 4, ctx->stream));
    CUDA_TRY(launch_set_bits(m->d, d_rows, d_cols, count, ctx->d_bad, ctx->stream));
    return check_bad(ctx, "cfpq_matrix_set_bits_device");
}

static int load_edges_impl(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, const uint32_t *from,
                           const uint32_t *label, const uint32_t *to, size_t nedges, const uint32_t *label_offsets,
                           const uint32_t *label_mats, uint32_t nlabels, bool on_device);

extern "C" int cfpq_load_edges(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, const uint32_t *from,
                               const uint32_t *label, const uint32_t *to, size_t nedges,
                               const uint32_t *label_offsets, const uint32_t *label_mats, uint32_t nlabels) {
    TRY(load_edges_impl(ctx, mats, nmats, from, label, to, nedges, label_offsets, label_mats, nlabels, false));
    return check_bad(ctx, "cfpq_load_edges");
}

extern "C" int cfpq_load_edges_device(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, const uint32_t *d_from,
                                      const uint32_t *d_label, const uint32_t *d_to, size_t nedges,
                                      const uint32_t *label_offsets, const uint32_t *label_mats, uint32_t nlabels) {
    return load_edges_impl(ctx, mats, nmats, d_from, d_label, d_to, nedges, label_offsets, label_mats, nlabels,
                           true);
}

extern "C" void *cfpq_ctx_stream(const cfpq_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }

// The device address of host array a[0..n) when all of it is pinned and
// mapped into this device's address space, else null.
static const uint32_t *mapped_host_array(const uint32_t *a, size_t n) {
    const uint32_t *ends[2] = {a, a + n - 1};
    const uint32_t *dev[2] = {nullptr, nullptr};
    for (int k = 0; k < 2; ++k) {
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, ends[k]) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        if (at.type != cudaMemoryTypeHost || !at.devicePointer) return nullptr;
        dev[k] = static_cast<const uint32_t *>(at.devicePointer);
    }
    return dev[1] == dev[0] + (n - 1) ? dev[0] : nullptr;
}

// Validates an edge list and stages it for the scatter: the small tables
// (matrix descriptors, label offsets, label -> matrices) on the device, host
// edge arrays copied (asynchronously) into the context's staging block --
// except with read_pinned_in_place, where arrays in pinned mapped host
// memory are read by the scatter kernel itself over the bus (the caller must
// keep them unchanged until the stream has run the kernel; *read_in_place
// tells which happened).  Fills the edge fields of *in; launches nothing.
// Nothing to scatter: in->nedges = 0.
static int prepare_edges(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, const uint32_t *from,
                         const uint32_t *label, const uint32_t *to, size_t nedges, const uint32_t *label_offsets,
                         const uint32_t *label_mats, uint32_t nlabels, bool on_device, ClosureInput *in,
                         bool read_pinned_in_place = false, bool *read_in_place = nullptr) {
    if (read_in_place) *read_in_place = false;
    in->nedges = 0;
    if ((nmats && !mats) || (nedges && (!from || !label || !to)) || (nlabels && (!label_offsets)))
        return set_error(CFPQ_ERR_INVALID, "null argument");
    if (nedges == 0 || nlabels == 0) return CFPQ_OK;
    const uint32_t nlm = label_offsets[nlabels];
    for (uint32_t l = 0; l < nlabels; ++l)
        if (label_offsets[l] > label_offsets[l + 1]) return set_error(CFPQ_ERR_INVALID, "label_offsets not sorted");
    if (nlm && !label_mats) return set_error(CFPQ_ERR_INVALID, "null label_mats");
    std::vector<DevMat> descs(nmats);
    for (size_t i = 0; i < nmats; ++i) {
        if (!mats[i]) return set_error(CFPQ_ERR_INVALID, "null matrix %zu", i);
        descs[i] = mats[i]->d;
    }
    for (uint32_t j = 0; j < nlm; ++j)
        if (label_mats[j] >= nmats) return set_error(CFPQ_ERR_INVALID, "label_mats[%u] out of range", j);
    // one staging block: descs | from | label | to | offsets | label_mats
    const size_t bd = nmats * sizeof(DevMat);
    const size_t be = nedges * 4;
    const size_t bo = (size_t)(nlabels + 1) * 4;
    const size_t bl = (size_t)(nlm ? nlm : 1) * 4;
    auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
    TRY(ctx->edge_buf.ensure(up(bd) + 3 * up(be) + up(bo) + up(bl)));
    char *base = ctx->edge_buf.as<char>();
    DevMat *d_desc = reinterpret_cast<DevMat *>(base);
    uint32_t *d_from = reinterpret_cast<uint32_t *>(base + up(bd));
    uint32_t *d_label = reinterpret_cast<uint32_t *>(base + up(bd) + up(be));
    uint32_t *d_to = reinterpret_cast<uint32_t *>(base + up(bd) + 2 * up(be));
    uint32_t *d_off = reinterpret_cast<uint32_t *>(base + up(bd) + 3 * up(be));
    uint32_t *d_lm = reinterpret_cast<uint32_t *>(base + up(bd) + 3 * up(be) + up(bo));
    // Small tables go through a pinned host block (copied with the call, so the
    // caller's arrays are free on return and the copy is truly asynchronous);
    // when they and the buffer layout equal the previous call's (the same
    // matrices and labels loaded again), the device copies are still there.
    std::vector<unsigned char> key(6 * sizeof(size_t) + bd + bo + (size_t)nlm * 4);
    {
        const size_t head[6] = {bd, be, bo, bl, (size_t)nlm, (size_t)(uintptr_t)ctx->edge_buf.p};
        unsigned char *k = key.data();
        memcpy(k, head, sizeof(head));
        memcpy(k + sizeof(head), descs.data(), bd);
        memcpy(k + sizeof(head) + bd, label_offsets, bo);
        if (nlm) memcpy(k + sizeof(head) + bd + bo, label_mats, (size_t)nlm * 4);
    }
    const bool tables_loaded = key == ctx->edge_tables_key;
    const size_t small = up(bd) + up(bo) + up(bl);
    if (!tables_loaded && ctx->h_small_cap < small) {
        if (ctx->h_small) cudaFreeHost(ctx->h_small);
        ctx->h_small = nullptr;
        ctx->h_small_cap = 0;
        CUDA_TRY(cudaMallocHost(&ctx->h_small, small));
        ctx->h_small_cap = small;
    }
    if (!tables_loaded) {
        ctx->edge_tables_key.clear();
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // previous user of h_small done
        char *hs = reinterpret_cast<char *>(ctx->h_small);
        memcpy(hs, descs.data(), bd);
        memcpy(hs + up(bd), label_offsets, bo);
        if (nlm) memcpy(hs + up(bd) + up(bo), label_mats, (size_t)nlm * 4);
        CUDA_TRY(cudaMemcpyAsync(d_desc, hs, bd, cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(cudaMemcpyAsync(d_off, hs + up(bd), bo, cudaMemcpyHostToDevice, ctx->stream));
        if (nlm)
            CUDA_TRY(cudaMemcpyAsync(d_lm, hs + up(bd) + up(bo), (size_t)nlm * 4, cudaMemcpyHostToDevice, ctx->stream));
        // host-edge loads overwrite the edge arrays only, never the tables
        ctx->edge_tables_key = std::move(key);
    }
    const uint32_t *m_from = nullptr, *m_label = nullptr, *m_to = nullptr;
    if (!on_device && read_pinned_in_place && (m_from = mapped_host_array(from, nedges)) &&
        (m_label = mapped_host_array(label, nedges)) && (m_to = mapped_host_array(to, nedges))) {
        d_from = const_cast<uint32_t *>(m_from);
        d_label = const_cast<uint32_t *>(m_label);
        d_to = const_cast<uint32_t *>(m_to);
        if (read_in_place) *read_in_place = true;
    } else if (on_device) {
        d_from = const_cast<uint32_t *>(from);
        d_label = const_cast<uint32_t *>(label);
        d_to = const_cast<uint32_t *>(to);
    } else {
        CUDA_TRY(cudaMemcpyAsync(d_from, from, be, cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(cudaMemcpyAsync(d_label, label, be, cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(cudaMemcpyAsync(d_to, to, be, cudaMemcpyHostToDevice, ctx->stream));
    }
    in->mats = d_desc;
    in->nmats = (uint32_t)nmats;
    in->nlabels = nlabels;
    in->from = d_from;
    in->label = d_label;
    in->to = d_to;
    in->nedges = nedges;
    in->off = d_off;
    in->lm = d_lm;
    in->nlm = nlm;
    in->bad = ctx->d_bad;
    return CFPQ_OK;
}

static int load_edges_impl(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, const uint32_t *from,
                           const uint32_t *label, const uint32_t *to, size_t nedges, const uint32_t *label_offsets,
                           const uint32_t *label_mats, uint32_t nlabels, bool on_device) {
    TRY(use_device(ctx));
    ClosureInput in;
    memset(&in, 0, sizeof(in));
    TRY(prepare_edges(ctx, mats, nmats, from, label, to, nedges, label_offsets, label_mats, nlabels, on_device, &in));
    if (!in.nedges) return CFPQ_OK;
    CUDA_TRY(cudaMemsetAsync(ctx->d_bad, 0, 4, ctx->stream));
    CUDA_TRY(launch_load_edges(in.mats, in.nmats, in.from, in.label, in.to, in.nedges, in.off, in.lm, in.nlabels,
                               in.nlm, ctx->d_bad, ctx->stream));
    return CFPQ_OK;
}

extern "C" int cfpq_matrix_set_diagonal(cfpq_ctx *ctx, cfpq_matrix *m) {
    TRY(use_device(ctx));
    if (!m) return set_error(CFPQ_ERR_INVALID, "null matrix");
    CUDA_TRY(launch_set_diag(m->d, ctx->stream));
    return CFPQ_OK;
}

extern "C" int cfpq_matrix_clear(cfpq_ctx *ctx, cfpq_matrix *m) {
    TRY(use_device(ctx));
    if (!m) return set_error(CFPQ_ERR_INVALID, "null matrix");
    CUDA_TRY(launch_clear_matrix(m->d, ctx->stream));
    return CFPQ_OK;
}

// The clear list of `count` matrices on the device (one unit per tile-row,
// MatRows prefix sums), re-sent only when it differs from the last one.
static int prepare_clear(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t count, ClosureInput *in) {
    in->clear_rows = 0;
    if (count == 0) return CFPQ_OK;
    if (!mats) return set_error(CFPQ_ERR_INVALID, "null matrix list");
    std::vector<MatRows> tab(count);
    uint32_t rows = 0;
    for (size_t i = 0; i < count; ++i) {
        if (!mats[i]) return set_error(CFPQ_ERR_INVALID, "matrix %zu is null", i);
        tab[i].m = mats[i]->d;
        tab[i].row_start = rows;
        tab[i].pad = 0;
        rows += mats[i]->d.T;
    }
    void *const before = ctx->clear_desc.p;
    TRY(ctx->clear_desc.ensure(count * sizeof(MatRows)));
    // the same list as the previous call (a prepared query cleared again):
    // its table is still on the device
    const unsigned char *tb = reinterpret_cast<const unsigned char *>(tab.data());
    std::vector<unsigned char> key(tb, tb + count * sizeof(MatRows));
    if (ctx->clear_desc.p != before || key != ctx->clear_desc_key) {
        ctx->clear_desc_key.clear();
        CUDA_TRY(cudaMemcpyAsync(ctx->clear_desc.p, tab.data(), count * sizeof(MatRows), cudaMemcpyHostToDevice,
                                 ctx->stream));
        ctx->clear_desc_key = std::move(key);
    }
    in->clear = ctx->clear_desc.as<MatRows>();
    in->nclear = (uint32_t)count;
    in->clear_rows = rows;
    return CFPQ_OK;
}

extern "C" int cfpq_matrices_clear(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t count) {
    TRY(use_device(ctx));
    ClosureInput in;
    memset(&in, 0, sizeof(in));
    TRY(prepare_clear(ctx, mats, count, &in));
    if (in.clear_rows) CUDA_TRY(launch_clear_rows(in.clear, in.nclear, in.clear_rows, ctx->stream));
    return CFPQ_OK;
}

extern "C" int cfpq_matrix_copy(cfpq_ctx *ctx, cfpq_matrix *dst, const cfpq_matrix *src) {
    TRY(use_device(ctx));
    if (!dst || !src) return set_error(CFPQ_ERR_INVALID, "null matrix");
    if (dst->d.n != src->d.n) return set_error(CFPQ_ERR_INVALID, "size mismatch %u vs %u", dst->d.n, src->d.n);
    if (dst->order != src->order) return set_error(CFPQ_ERR_INVALID, "matrices have different vertex orders");
    if (dst == src) return CFPQ_OK;
    CUDA_TRY(launch_copy_matrix(dst->d, src->d, ctx->stream));
    return CFPQ_OK;
}

extern "C" int cfpq_matrix_upload_rows(cfpq_ctx *ctx, cfpq_matrix *m, const uint64_t *host_rows) {
    TRY(use_device(ctx));
    if (!m || (!host_rows && m->d.n)) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (m->d.n == 0) return CFPQ_OK;
    const size_t words = (size_t)m->d.n * m->d.T;
    TRY(ctx->stage.ensure(words * 8));
    CUDA_TRY(cudaMemcpyAsync(ctx->stage.p, host_rows, words * 8, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(launch_rows_to_tiles(m->d, ctx->stage.as<uint64_t>(), ctx->stream));
    return sync_and_check(ctx);
}

extern "C" int cfpq_matrix_download_rows(cfpq_ctx *ctx, const cfpq_matrix *m, uint64_t *host_rows) {
    TRY(use_device(ctx));
    if (!m || (!host_rows && m->d.n)) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (m->d.n == 0) return CFPQ_OK;
    const size_t words = (size_t)m->d.n * m->d.T;
    TRY(ctx->stage.ensure(words * 8));
    CUDA_TRY(launch_tiles_to_rows(m->d, ctx->stage.as<uint64_t>(), ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(host_rows, ctx->stage.p, words * 8, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_and_check(ctx);
}

extern "C" int cfpq_matrix_tile_stats(cfpq_ctx *ctx, const cfpq_matrix *m, uint32_t *occ_out, uint32_t *nnz_out) {
    TRY(use_device(ctx));
    if (!m) return set_error(CFPQ_ERR_INVALID, "null matrix");
    if (m->d.T == 0) return CFPQ_OK;
    if (occ_out)
        CUDA_TRY(cudaMemcpyAsync(occ_out, m->d.occ, (size_t)m->d.T * m->d.ow * 4, cudaMemcpyDeviceToHost, ctx->stream));
    if (nnz_out)
        CUDA_TRY(cudaMemcpyAsync(nnz_out, m->d.nnz, (size_t)m->d.T * m->d.T * 4, cudaMemcpyDeviceToHost, ctx->stream));
    return sync_and_check(ctx);
}

// Result buffers for nm matrices and `blocks` hash blocks: the pinned h_hash
// (written by the kernel through its mapping when the device can map it,
// else copied from d_hash), the per-block partial sums and the ticket.
static int ensure_hash_buffers(cfpq_ctx *ctx, size_t nm, size_t blocks) {
    if (ctx->d_hash_cap < nm) {
        if (ctx->d_hash) cudaFree(ctx->d_hash);
        if (ctx->h_hash) cudaFreeHost(ctx->h_hash);
        ctx->d_hash = nullptr;
        ctx->h_hash = ctx->h_hash_dev = nullptr;
        ctx->d_hash_cap = ctx->h_hash_cap = 0;
        CUDA_TRY(cudaMalloc(&ctx->d_hash, nm * 2 * sizeof(unsigned long long)));
        CUDA_TRY(cudaMallocHost(&ctx->h_hash, nm * 2 * sizeof(unsigned long long)));
        if (cudaHostGetDevicePointer(reinterpret_cast<void **>(&ctx->h_hash_dev), ctx->h_hash, 0) != cudaSuccess) {
            ctx->h_hash_dev = nullptr;
            cudaGetLastError();
        }
        ctx->d_hash_cap = ctx->h_hash_cap = nm;
    }
    if (ctx->d_hash_part_cap < blocks) {
        if (ctx->d_hash_part) cudaFree(ctx->d_hash_part);
        ctx->d_hash_part = nullptr;
        ctx->d_hash_part_cap = 0;
        CUDA_TRY(cudaMalloc(&ctx->d_hash_part, blocks * 2 * sizeof(unsigned long long)));
        ctx->d_hash_part_cap = blocks;
    }
    if (!ctx->d_hash_ticket) {
        CUDA_TRY(cudaMalloc(&ctx->d_hash_ticket, sizeof(uint32_t)));
        CUDA_TRY(cudaMemsetAsync(ctx->d_hash_ticket, 0, sizeof(uint32_t), ctx->stream));
    }
    return CFPQ_OK;
}

// Hash launches of several matrices (one kernel per kHashBatch matrices, one
// block per tile-row); their (hash, count) pairs land in the pinned h_hash
// with no copy after the kernel when h_hash is mapped.
static int enqueue_hash_many(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats) {
    size_t blocks = 0;
    for (size_t i0 = 0; i0 < nmats; i0 += kHashBatch) {
        size_t b = 0;
        for (size_t i = i0; i < nmats && i < i0 + kHashBatch; ++i) {
            if (!mats[i]) return set_error(CFPQ_ERR_INVALID, "null matrix %zu", i);
            b += mats[i]->d.T;
        }
        blocks = std::max(blocks, b);
    }
    TRY(ensure_hash_buffers(ctx, nmats, blocks));
    unsigned long long *const out = ctx->h_hash_dev ? ctx->h_hash_dev : ctx->d_hash;
    for (size_t i0 = 0; i0 < nmats; i0 += kHashBatch) {
        HashBatch hb;
        memset(&hb, 0, sizeof(hb));
        for (size_t i = i0; i < nmats && i < i0 + kHashBatch; ++i) {
            PowTables pt;
            TRY(get_pow_tables(ctx, mats[i], &pt));
            const uint32_t k = hb.count++;
            hb.m[k] = mats[i]->d;
            hb.nib11[k] = pt.d_nib11;
            hb.pow13[k] = pt.d_pow13;
            hb.start[k + 1] = hb.start[k] + mats[i]->d.T;  // one block per tile-row
        }
        if (hb.start[hb.count] == 0) {  // matrices of size 0 only: their lines are (0, 0)
            if (ctx->h_hash_dev) memset(ctx->h_hash + 2 * i0, 0, 2 * sizeof(unsigned long long) * hb.count);
            else CUDA_TRY(cudaMemsetAsync(ctx->d_hash + 2 * i0, 0, 2 * sizeof(unsigned long long) * hb.count,
                                          ctx->stream));
            continue;
        }
        CUDA_TRY(launch_hash_lines(hb, ctx->d_hash_part, ctx->d_hash_ticket, out + 2 * i0, ctx->stream));
    }
    if (!ctx->h_hash_dev)
        CUDA_TRY(cudaMemcpyAsync(ctx->h_hash, ctx->d_hash, nmats * 2 * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    return CFPQ_OK;
}

extern "C" int cfpq_hash_count_many(cfpq_ctx *ctx, cfpq_matrix *const *mats, size_t nmats, uint64_t *hashes,
                                    uint64_t *counts) {
    TRY(use_device(ctx));
    if (nmats && (!mats || !hashes || !counts)) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (nmats == 0) return CFPQ_OK;
    TRY(enqueue_hash_many(ctx, mats, nmats));
    TRY(sync_and_check(ctx));
    for (size_t i = 0; i < nmats; ++i) {
        hashes[i] = ctx->h_hash[2 * i] % 1000000007ULL;
        counts[i] = ctx->h_hash[2 * i + 1];
    }
    return CFPQ_OK;
}

extern "C" int cfpq_matrix_hash_count(cfpq_ctx *ctx, const cfpq_matrix *m, uint64_t *hash, uint64_t *count) {
    if (!m || !hash || !count) return set_error(CFPQ_ERR_INVALID, "null argument");
    cfpq_matrix *mm = const_cast<cfpq_matrix *>(m);
    return cfpq_hash_count_many(ctx, &mm, 1, hash, count);
}

extern "C" int cfpq_matrix_count(cfpq_ctx *ctx, const cfpq_matrix *m, uint64_t *count) {
    uint64_t h = 0;
    return cfpq_matrix_hash_count(ctx, m, &h, count);
}

// ---------------------------------------------------------------------------
// one product (add_mul)

static int read_flag(cfpq_ctx *ctx, uint32_t *dflag, int *changed) {
    CUDA_TRY(cudaMemcpyAsync(ctx->h_flag, dflag, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *changed = ctx->h_flag[0] != 0;
    return CFPQ_OK;
}

static int launch_products(cfpq_ctx *ctx, size_t list_cap, bool lop3, bool m4r, uint32_t *qchanged,
                           BufCounters *cnts, cudaStream_t s);

// A tensor-core product term of a closure plan.
struct TcProduct {
    uint32_t index, T, row_start, rows;
};

// One tensor-core product: plan its items, run the tensor-core kernel, close
// the item list.  With a choice array the plan emits nothing (and the kernel
// finds no items) unless this iteration's variant of the product is TC.
static int launch_tc_product(cfpq_ctx *ctx, const TcProduct &tp, uint32_t nprods, size_t list_cap,
                             uint32_t *prod_seen, uint32_t *qchanged, const uint8_t *choice, BufCounters *cnts,
                             cudaStream_t s) {
    const ProdDesc *pr = ctx->prods.as<ProdDesc>();
    const MatSlot *sl = ctx->slots.as<MatSlot>();
    CUDA_TRY(launch_plan(pr, nprods, tp.row_start, tp.row_start + tp.rows, sl, ctx->d_st, ctx->items.as<uint64_t>(),
                         list_cap, product_lop3_tiles_per_block(), prod_seen, 1, choice, s));
    CUDA_TRY(launch_product_tc(pr, sl, ctx->d_st, ctx->items.as<uint64_t>(), list_cap, qchanged, ctx->tc_grid, cnts,
                               s));
    CUDA_TRY(launch_reset_list(ctx->d_st, 2, s));
    return CFPQ_OK;
}

// Enqueue c |= a * b with a tiled variant (operands must not alias c); with
// a tile-row range [ti0, ti1) only those output tile-rows (word-level
// variants; tensor-core products always cover the whole matrix).
static int enqueue_tiled_product(cfpq_ctx *ctx, const DevMat &a, const DevMat &b, const DevMat &c, int variant,
                                 uint32_t ti0 = 0, uint32_t ti1 = 0xFFFFFFFFu) {
    const uint32_t T = a.T;
    ti1 = std::min(ti1, T);
    const int tpb = product_lop3_tiles_per_block();
    MatSlot hs[3];
    memset(hs, 0, sizeof(hs));
    hs[0].cur = a;
    hs[1].cur = b;
    hs[2].cur = c;
    ProdDesc pd;
    memset(&pd, 0, sizeof(pd));
    pd.head = 2;
    pd.pslot = 0;
    pd.qslot = 1;
    pd.T = T;
    pd.n = a.n;
    pd.variant = (uint8_t)variant;
    const size_t cap = std::max<size_t>(item_capacity(T, tpb), 1);
    ctx->tables_owner = 0;
    TRY(ctx->slots.ensure(sizeof(hs)));
    TRY(ctx->prods.ensure(sizeof(pd)));
    TRY(ctx->items.ensure(3 * cap * 8));
    ctx->items_clean_words = 0;
    IterState st;
    memset(&st, 0, sizeof(st));
    st.iter = 1;
    st.active = 1;
    *ctx->h_st = st;
    CUDA_TRY(cudaMemcpyAsync(ctx->slots.p, hs, sizeof(hs), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(ctx->prods.p, &pd, sizeof(pd), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(ctx->d_st, ctx->h_st, sizeof(IterState), cudaMemcpyHostToDevice, ctx->stream));
    if (variant == CFPQ_VARIANT_TC) {
        return launch_tc_product(ctx, TcProduct{0, T, 0, (T + 3) / 4}, 1, cap, nullptr, nullptr, nullptr, nullptr,
                                 ctx->stream);
    }
    CUDA_TRY(launch_plan(ctx->prods.as<ProdDesc>(), 1, ti0, ti1, ctx->slots.as<MatSlot>(), ctx->d_st,
                         ctx->items.as<uint64_t>(), cap, tpb, nullptr, 0, nullptr, ctx->stream));
    TRY(launch_products(ctx, cap, variant == CFPQ_VARIANT_LOP3, variant == CFPQ_VARIANT_M4R, nullptr, nullptr,
                        ctx->stream));
    return CFPQ_OK;
}

// Word-level product kernels of one closure iteration: one launch per item
// list in use.
static int launch_products(cfpq_ctx *ctx, size_t list_cap, bool lop3, bool m4r, uint32_t *qchanged,
                           BufCounters *cnts, cudaStream_t s) {
    if (lop3)
        CUDA_TRY(launch_product_tiled(0, ctx->prods.as<ProdDesc>(), ctx->slots.as<MatSlot>(), ctx->d_st,
                                      ctx->items.as<uint64_t>(), list_cap, qchanged, ctx->lop3_grid, cnts, s));
    if (m4r)
        CUDA_TRY(launch_product_tiled(1, ctx->prods.as<ProdDesc>(), ctx->slots.as<MatSlot>(), ctx->d_st,
                                      ctx->items.as<uint64_t>(), list_cap, qchanged, ctx->m4r_grid, cnts, s));
    return CFPQ_OK;
}

static int add_mul_impl(cfpq_ctx *ctx, cfpq_matrix *c, const cfpq_matrix *a, const cfpq_matrix *b, int variant,
                        int *changed, uint32_t ti0, uint32_t ti1);

extern "C" int cfpq_add_mul(cfpq_ctx *ctx, cfpq_matrix *c, const cfpq_matrix *a, const cfpq_matrix *b, int variant,
                            int *changed) {
    return add_mul_impl(ctx, c, a, b, variant, changed, 0, 0xFFFFFFFFu);
}

extern "C" int cfpq_add_mul_rows(cfpq_ctx *ctx, cfpq_matrix *c, const cfpq_matrix *a, const cfpq_matrix *b,
                                 int variant, uint32_t row_begin, uint32_t row_end, int *changed) {
    if (!c || !a || !b || !changed) return set_error(CFPQ_ERR_INVALID, "null argument");
    const uint32_t n = c->d.n;
    if (row_begin > row_end || row_end > n || row_begin % 64 || (row_end % 64 && row_end != n))
        return set_error(CFPQ_ERR_INVALID, "row range [%u, %u) of an n = %u matrix: bounds must be multiples of 64 "
                         "(the end may be n)", row_begin, row_end, n);
    if (variant == CFPQ_VARIANT_AUTO) variant = CFPQ_VARIANT_LOP3;
    if (variant != CFPQ_VARIANT_LOP3 && variant != CFPQ_VARIANT_M4R)
        return set_error(CFPQ_ERR_UNSUPPORTED, "row-range products run the LOP3 or Four Russians variant");
    if (c->order || a->order || b->order)
        return set_error(CFPQ_ERR_UNSUPPORTED, "row-range products need matrices without a vertex order");
    *changed = 0;
    if (row_begin == row_end) return CFPQ_OK;
    return add_mul_impl(ctx, c, a, b, variant, changed, row_begin / 64, (row_end + 63) / 64);
}

static int add_mul_impl(cfpq_ctx *ctx, cfpq_matrix *c, const cfpq_matrix *a, const cfpq_matrix *b, int variant,
                        int *changed, uint32_t ti0, uint32_t ti1) {
    TRY(use_device(ctx));
    if (!c || !a || !b || !changed) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (a->d.n != c->d.n || b->d.n != c->d.n)
        return set_error(CFPQ_ERR_INVALID, "size mismatch (%u, %u, %u)", c->d.n, a->d.n, b->d.n);
    if (a->order != c->order || b->order != c->order)
        return set_error(CFPQ_ERR_INVALID, "operands have different vertex orders");
    *changed = 0;
    if (c->d.n == 0) return CFPQ_OK;
    if (variant == CFPQ_VARIANT_AUTO) variant = CFPQ_VARIANT_LOP3;
    const bool alias = (a == c) || (b == c);
    if (variant == CFPQ_VARIANT_PLAIN) {
        CUDA_TRY(cudaMemsetAsync(ctx->d_flag, 0, 4, ctx->stream));
        if (alias) {
            cfpq_matrix *tmp = nullptr;
            TRY(pool_take(ctx, c->d.n, &tmp));
            CUDA_TRY(launch_plain_product(a->d, b->d, tmp->d, 1, ctx->d_flag, ctx->stream));
            CUDA_TRY(launch_merge_or(c->d, tmp->d, ctx->d_flag, ctx->stream));
            TRY(pool_give(ctx, tmp, true));
        } else {
            CUDA_TRY(launch_plain_product(a->d, b->d, c->d, 0, ctx->d_flag, ctx->stream));
        }
        return read_flag(ctx, ctx->d_flag, changed);
    }
    if (variant != CFPQ_VARIANT_LOP3 && variant != CFPQ_VARIANT_M4R && variant != CFPQ_VARIANT_TC)
        return set_error(CFPQ_ERR_UNSUPPORTED, "variant %d is not available for add_mul", variant);
    if (variant == CFPQ_VARIANT_TC && !ctx->tc_grid)
        return set_error(CFPQ_ERR_UNSUPPORTED, "tensor-core variant unavailable (needs one CTA per SM)");
    // Snapshot semantics: operands that alias c are read from a copy.
    cfpq_matrix *ca = nullptr, *cb = nullptr;
    DevMat da = a->d, db = b->d;
    if (a == c) {
        TRY(pool_take(ctx, c->d.n, &ca));
        CUDA_TRY(launch_copy_matrix(ca->d, a->d, ctx->stream));
        da = ca->d;
    }
    if (b == c) {
        if (a == b) {
            db = da;
        } else {
            TRY(pool_take(ctx, c->d.n, &cb));
            CUDA_TRY(launch_copy_matrix(cb->d, b->d, ctx->stream));
            db = cb->d;
        }
    }
    TRY(enqueue_tiled_product(ctx, da, db, c->d, variant, ti0, ti1));
    CUDA_TRY(cudaMemcpyAsync(ctx->h_st, ctx->d_st, sizeof(IterState), cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (ca) TRY(pool_give(ctx, ca, true));
    if (cb) TRY(pool_give(ctx, cb, true));
    if (ctx->h_st->error) return set_error(CFPQ_ERR_TIMEOUT, "a bounded device wait gave up (product kernel)");
    *changed = ctx->h_st->changed != 0;
    return CFPQ_OK;
}

// ---------------------------------------------------------------------------
// row blocks (multi-GPU row-block closure)

// Tile-rows [ti0, ti1) of a row range; false if the bounds are invalid.
static bool block_tiles(const cfpq_matrix *m, uint32_t row_begin, uint32_t row_end, uint32_t *ti0, uint32_t *ti1) {
    const uint32_t n = m->d.n;
    if (row_begin > row_end || row_end > n || row_begin % 64 || (row_end % 64 && row_end != n)) return false;
    *ti0 = row_begin / 64;
    *ti1 = (row_end + 63) / 64;
    return true;
}

extern "C" size_t cfpq_matrix_block_bytes(const cfpq_matrix *m, uint32_t row_begin, uint32_t row_end) {
    uint32_t ti0, ti1;
    if (!m || !block_tiles(m, row_begin, row_end, &ti0, &ti1)) return 0;
    const size_t tr = ti1 - ti0, T = m->d.T;
    return tr * T * 512 + tr * m->d.ow * 4 + tr * T * 4;
}

// Copies of the three contiguous ranges of a block (bits, occupancy words,
// tile populations) between a matrix and a packed buffer (device or host:
// cudaMemcpyDefault).
static int block_copy(cfpq_ctx *ctx, cfpq_matrix *m, uint32_t row_begin, uint32_t row_end, void *buf, bool to_buf) {
    TRY(use_device(ctx));
    uint32_t ti0, ti1;
    if (!m || !buf) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (!block_tiles(m, row_begin, row_end, &ti0, &ti1))
        return set_error(CFPQ_ERR_INVALID, "row range [%u, %u) of an n = %u matrix: bounds must be multiples of 64 "
                         "(the end may be n)", row_begin, row_end, m->d.n);
    if (m->order) return set_error(CFPQ_ERR_UNSUPPORTED, "row blocks of matrices with a vertex order");
    const size_t tr = ti1 - ti0, T = m->d.T, ow = m->d.ow;
    if (!tr) return CFPQ_OK;
    char *p = static_cast<char *>(buf);
    void *dev[3] = {m->d.bits + (size_t)ti0 * T * 64, m->d.occ + (size_t)ti0 * ow, m->d.nnz + (size_t)ti0 * T};
    const size_t bytes[3] = {tr * T * 512, tr * ow * 4, tr * T * 4};
    for (int k = 0; k < 3; ++k) {
        if (to_buf)
            CUDA_TRY(cudaMemcpyAsync(p, dev[k], bytes[k], cudaMemcpyDefault, ctx->stream));
        else
            CUDA_TRY(cudaMemcpyAsync(dev[k], p, bytes[k], cudaMemcpyDefault, ctx->stream));
        p += bytes[k];
    }
    return CFPQ_OK;
}

extern "C" int cfpq_matrix_export_block(cfpq_ctx *ctx, const cfpq_matrix *m, uint32_t row_begin, uint32_t row_end,
                                        void *dst) {
    return block_copy(ctx, const_cast<cfpq_matrix *>(m), row_begin, row_end, dst, true);
}

extern "C" int cfpq_matrix_import_block(cfpq_ctx *ctx, cfpq_matrix *m, uint32_t row_begin, uint32_t row_end,
                                        const void *src) {
    return block_copy(ctx, m, row_begin, row_end, const_cast<void *>(src), false);
}

extern "C" int cfpq_matrix_delta(cfpq_ctx *ctx, cfpq_matrix *delta, const cfpq_matrix *cur, cfpq_matrix *prev) {
    TRY(use_device(ctx));
    if (!delta || !cur || !prev) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (delta->d.n != cur->d.n || prev->d.n != cur->d.n)
        return set_error(CFPQ_ERR_INVALID, "size mismatch (%u, %u, %u)", delta->d.n, cur->d.n, prev->d.n);
    if (delta == cur || delta == prev || prev == cur)
        return set_error(CFPQ_ERR_INVALID, "delta, current and previous must be three different matrices");
    if (delta->order != cur->order || prev->order != cur->order)
        return set_error(CFPQ_ERR_INVALID, "matrices with different vertex orders");
    CUDA_TRY(launch_delta_snapshot(delta->d, cur->d, prev->d, ctx->stream));
    return CFPQ_OK;
}

// ---------------------------------------------------------------------------
// closure

namespace {

struct QueryIn {
    const cfpq_rule *rules;
    size_t nrules;
    cfpq_matrix *const *mats;
    size_t nmats;
};

struct ClosurePlan {
    std::vector<MatSlot> slots;
    std::vector<ProdDesc> prods;
    std::vector<cfpq_matrix *> deltas;
    uint32_t slot_rows = 0, prod_rows = 0;
    size_t item_cap = 0;  // per item list
    bool uses_lop3 = false, uses_m4r = false, uses_tc = false;
    std::vector<TcProduct> tc_prods;
    std::vector<TcRows> tc_rows;  // the same for the grouped tensor-core plan (k_plan_tc)
    uint32_t tc_groups = 0;       // groups of 4 tile-rows over all tensor-core-capable products
    uint32_t tc_max_T = 0;
    bool auto_select = false;     // variants chosen on the device every iteration
    uint8_t fixed_variant = 0;    // otherwise: every product's variant
    std::vector<uint8_t> tc_ok;   // per product: has a tensor-core launch sequence
    std::vector<QueryRange> qranges;  // per query: its plan rows, slot rows, slots and products
};


}  // namespace

// The plan of the last closure, reused while the next closure has the same
// rules, matrices and variant (a prepared query run again): its delta buffers
// stay attached, and its device tables are re-sent only if something else
// used the table buffers in between.
struct PlanCache {
    bool valid = false;
    uint64_t id = 0;
    std::vector<uint64_t> key;
    ClosurePlan pl;
};

// Frees the cached plan at context destruction (deltas go to the pool first).
static void free_plan_cache(cfpq_ctx *ctx) {
    if (!ctx->pcache) return;
    for (auto *m : ctx->pcache->pl.deltas) ctx->pool.push_back(m);
    delete ctx->pcache;
    ctx->pcache = nullptr;
}

static int validate_query(const QueryIn &q, size_t qi) {
    if (q.nmats && !q.mats) return set_error(CFPQ_ERR_INVALID, "query %zu: null matrix array", qi);
    if (q.nrules && !q.rules) return set_error(CFPQ_ERR_INVALID, "query %zu: null rule array", qi);
    uint32_t n = 0;
    for (size_t i = 0; i < q.nmats; ++i) {
        if (!q.mats[i]) return set_error(CFPQ_ERR_INVALID, "query %zu: null matrix %zu", qi, i);
        if (i == 0) n = q.mats[i]->d.n;
        if (q.mats[i]->d.n != n)
            return set_error(CFPQ_ERR_INVALID, "query %zu: matrices of different sizes (%u vs %u)", qi, n,
                             q.mats[i]->d.n);
        if (q.mats[i]->order != q.mats[0]->order)
            return set_error(CFPQ_ERR_INVALID, "query %zu: matrices with different vertex orders", qi);
        for (size_t j = 0; j < i; ++j)
            if (q.mats[j] == q.mats[i])
                return set_error(CFPQ_ERR_INVALID, "query %zu: matrix %zu repeated at %zu", qi, i, j);
    }
    for (size_t r = 0; r < q.nrules; ++r) {
        const cfpq_rule &ru = q.rules[r];
        if (ru.head >= q.nmats || ru.body1 >= q.nmats || ru.body2 >= q.nmats)
            return set_error(CFPQ_ERR_INVALID, "query %zu: rule %zu refers to a matrix out of range", qi, r);
    }
    return CFPQ_OK;
}

// Largest tile count (n / 64) of a single closure whose persistent kernel
// merges item results without reading C first.
static constexpr uint32_t kDirectMergeMaxTiles = 256;

static int build_plan(cfpq_ctx *ctx, const std::vector<QueryIn> &qs, int variant, ClosurePlan *pl) {
    const int tpb = product_lop3_tiles_per_block();
    // AUTO with a selector: chosen per term and iteration among the allowed
    // variants; else one variant for every term (PLAIN and fixed-mode AUTO
    // run the LOP3 kernel)
    const uint32_t allowed = ctx->sel.allowed & ((1u << CFPQ_VARIANT_LOP3) | (1u << CFPQ_VARIANT_M4R) |
                                                 (ctx->tc_grid ? 1u << CFPQ_VARIANT_TC : 0u));
    uint32_t max_T = 0;
    for (const QueryIn &q : qs)
        if (q.nmats && q.nrules) max_T = std::max(max_T, q.mats[0]->d.T);
    // a single small query is latency-bound: selection costs more than it gains
    pl->auto_select = variant == CFPQ_VARIANT_AUTO && ctx->sel.mode != CFPQ_SELECT_FIXED &&
                      (allowed & ~(1u << CFPQ_VARIANT_LOP3)) != 0 && (qs.size() > 1 || max_T >= ctx->sel.min_tiles);
    pl->fixed_variant = (uint8_t)(variant == CFPQ_VARIANT_M4R || variant == CFPQ_VARIANT_TC ? variant
                                                                                           : CFPQ_VARIANT_LOP3);
    const bool tc_auto = (allowed & (1u << CFPQ_VARIANT_TC)) != 0;
    if (pl->auto_select) {
        pl->uses_lop3 = (allowed & (1u << CFPQ_VARIANT_LOP3)) != 0;
        pl->uses_m4r = (allowed & (1u << CFPQ_VARIANT_M4R)) != 0;
        if (!pl->uses_lop3 && !pl->uses_m4r) pl->uses_lop3 = true;  // the heuristic's last resort
    } else {
        pl->uses_lop3 = pl->fixed_variant == CFPQ_VARIANT_LOP3;
        pl->uses_m4r = pl->fixed_variant == CFPQ_VARIANT_M4R;
    }
    for (size_t qi = 0; qi < qs.size(); ++qi) {
        const QueryIn &q = qs[qi];
        const uint32_t base = (uint32_t)pl->slots.size();
        QueryRange qrange;
        qrange.prow0 = pl->prod_rows;
        qrange.srow0 = pl->slot_rows;
        qrange.slot0 = base;
        qrange.prod0 = (uint32_t)pl->prods.size();
        for (size_t i = 0; i < q.nmats; ++i) {
            MatSlot s;
            memset(&s, 0, sizeof(s));
            s.cur = q.mats[i]->d;
            s.query = (uint32_t)qi;
            s.row_start = pl->slot_rows;
            for (int k = 0; k < 2; ++k) {
                cfpq_matrix *dm = nullptr;
                TRY(pool_take(ctx, s.cur.n, &dm));
                pl->deltas.push_back(dm);
                s.dlt[k] = dm->d;
            }
            pl->slot_rows += s.cur.T;
            pl->slots.push_back(s);
        }
        const uint32_t T = q.nmats ? q.mats[0]->d.T : 0, n = q.nmats ? q.mats[0]->d.n : 0;
        for (size_t r = 0; r < q.nrules && T; ++r) {
            for (uint8_t term = 0; term < 2; ++term) {
                ProdDesc pd;
                memset(&pd, 0, sizeof(pd));
                pd.head = base + q.rules[r].head;
                pd.pslot = base + q.rules[r].body1;
                pd.qslot = base + q.rules[r].body2;
                pd.p_delta = term == 0;
                pd.q_delta = term == 1;
                pd.term = term;
                pd.variant = pl->auto_select ? (uint8_t)CFPQ_VARIANT_AUTO : pl->fixed_variant;
                pd.query = (uint32_t)qi;
                pd.rule = (uint32_t)r;
                pd.T = T;
                pd.n = n;
                // plan rows: T tile-rows for the word-level kernels; a term that
                // may run on tensor cores also plans ceil(T/4) groups of 4
                // tile-rows from the same start in its own launch
                pd.row_start = pl->prod_rows;
                const bool tc = pl->auto_select ? tc_auto && T >= ctx->sel.tc_min_tiles
                                                : pl->fixed_variant == CFPQ_VARIANT_TC;
                if (tc) {
                    pl->tc_prods.push_back(TcProduct{(uint32_t)pl->prods.size(), T, pl->prod_rows, (T + 3) / 4});
                    pl->tc_max_T = std::max(pl->tc_max_T, T);
                }
                pl->tc_ok.push_back(tc ? 1 : 0);
                pl->prod_rows += T;
                pl->item_cap += item_capacity(T, tpb);
                pl->prods.push_back(pd);
            }
        }
        qrange.nprow = pl->prod_rows - qrange.prow0;
        qrange.nsrow = pl->slot_rows - qrange.srow0;
        qrange.nslot = (uint32_t)pl->slots.size() - qrange.slot0;
        qrange.nprod = (uint32_t)pl->prods.size() - qrange.prod0;
        pl->qranges.push_back(qrange);
    }
    pl->item_cap = std::max<size_t>(pl->item_cap, 1);
    pl->uses_tc = !pl->tc_prods.empty();
    for (const TcProduct &tp : pl->tc_prods) {
        pl->tc_rows.push_back(TcRows{tp.index, tp.row_start, pl->tc_groups, 0});
        pl->tc_groups += tp.rows;
    }
    if (pl->prods.size() > kMaxItemProducts)
        return set_error(CFPQ_ERR_INVALID, "%zu rule products in one closure (at most %u)", pl->prods.size(),
                         kMaxItemProducts);
    return CFPQ_OK;
}

// Cache key of a closure: variant, and per query its rules and the device
// layout of its matrices.
static void plan_key(const cfpq_ctx *ctx, const std::vector<QueryIn> &qs, int variant,
                     std::vector<uint64_t> *key) {
    key->clear();
    key->push_back(((uint64_t)(uint32_t)variant << 32) | (uint64_t)qs.size());
    key->push_back(((uint64_t)(uint32_t)ctx->sel.mode << 40) | ((uint64_t)ctx->sel.allowed << 32) |
                   ctx->sel.tc_min_tiles);
    key->push_back(ctx->sel.min_tiles);
    for (const QueryIn &q : qs) {
        key->push_back(((uint64_t)q.nrules << 32) | (uint64_t)q.nmats);
        for (size_t r = 0; r < q.nrules; ++r)
            key->push_back(((uint64_t)q.rules[r].head << 42) ^ ((uint64_t)q.rules[r].body1 << 21) ^
                           (uint64_t)q.rules[r].body2);
        for (size_t i = 0; i < q.nmats; ++i) {
            const DevMat &d = q.mats[i]->d;
            key->push_back((uint64_t)(uintptr_t)d.bits);
            key->push_back((uint64_t)(uintptr_t)d.occ ^ ((uint64_t)(uintptr_t)d.nnz << 1));
            key->push_back((uint64_t)(uintptr_t)d.perm ^ ((uint64_t)d.n << 40));
        }
    }
}

// Forget the cached plan; its deltas go back to the pool (cleared if dirty).
static void drop_plan_cache(cfpq_ctx *ctx, bool dirty) {
    if (!ctx->pcache) return;
    PlanCache &pc = *ctx->pcache;
    for (auto *m : pc.pl.deltas) pool_give(ctx, m, dirty);
    pc.pl = ClosurePlan();
    pc.key.clear();
    pc.valid = false;
}

// Buffer counters of a closure: kept (and read) only when the selector runs.
static BufCounters *closure_counters(cfpq_ctx *ctx, const ClosurePlan &) {
    return ctx->cnts_on ? ctx->cnts.as<BufCounters>() : nullptr;
}

// Plan of one iteration; in AUTO closures the planner also chooses every
// term's variant (PlanSelect).
static int enqueue_select_plan(cfpq_ctx *ctx, const ClosurePlan &pl, const QueryTrack &qt, cudaStream_t s) {
    const PlanSelect ps = {ctx->d_sel.as<SelectorParams>(), ctx->cnts.as<BufCounters>(), ctx->tc_ok.as<uint8_t>(),
                           ctx->choice.as<uint8_t>(), ctx->sel_log_iters ? ctx->sel_log.as<SelLogRow>() : nullptr,
                           ctx->sel_log_iters};
    CUDA_TRY(launch_plan(ctx->prods.as<ProdDesc>(), (uint32_t)pl.prods.size(), 0, pl.prod_rows,
                         ctx->slots.as<MatSlot>(), ctx->d_st, ctx->items.as<uint64_t>(), pl.item_cap,
                         product_lop3_tiles_per_block(), ctx->prod_seen.as<uint32_t>(), 0, ctx->choice.as<uint8_t>(),
                         s, pl.auto_select ? &ps : nullptr, qt.last_iter));
    return CFPQ_OK;
}

// Product kernels of one iteration: the word-level lists, then the tensor-core
// sequence of every term that may run on tensor cores.
static int enqueue_products(cfpq_ctx *ctx, const ClosurePlan &pl, const QueryTrack &qt, cudaStream_t s) {
    BufCounters *cnts = closure_counters(ctx, pl);
    TRY(launch_products(ctx, pl.item_cap, pl.uses_lop3, pl.uses_m4r, qt.changed, cnts, s));
    if (!pl.tc_prods.empty()) {
        // every tensor-core product of the iteration together: one plan
        // launch, one tensor-core launch over all their items, one list reset
        const ProdDesc *pr = ctx->prods.as<ProdDesc>();
        const MatSlot *sl = ctx->slots.as<MatSlot>();
        CUDA_TRY(launch_plan_tc(pr, (uint32_t)pl.prods.size(), ctx->tc_rows.as<TcRows>(),
                                (uint32_t)pl.tc_rows.size(), pl.tc_groups, sl, ctx->d_st, ctx->items.as<uint64_t>(),
                                pl.item_cap, product_lop3_tiles_per_block(), ctx->prod_seen.as<uint32_t>(),
                                ctx->choice.as<uint8_t>(), s, qt.last_iter));
        CUDA_TRY(launch_product_tc(pr, sl, ctx->d_st, ctx->items.as<uint64_t>(), pl.item_cap, qt.changed,
                                   ctx->tc_grid, cnts, s));
        CUDA_TRY(launch_reset_list(ctx->d_st, 2, s));
    }
    return CFPQ_OK;
}

static int enqueue_iteration(cfpq_ctx *ctx, const ClosurePlan &pl, const QueryTrack &qt,
                             cudaGraphConditionalHandle handle, int use_handle) {
    TRY(enqueue_select_plan(ctx, pl, qt, ctx->stream));
    TRY(enqueue_products(ctx, pl, qt, ctx->stream));
    CUDA_TRY(launch_advance_end(ctx->slots.as<MatSlot>(), (uint32_t)pl.slots.size(), pl.slot_rows, ctx->d_st, qt,
                                handle, use_handle, closure_counters(ctx, pl), ctx->stream));
    return CFPQ_OK;
}

// One iteration with every phase bracketed by events (profiling mode).
static int enqueue_iteration_timed(cfpq_ctx *ctx, const ClosurePlan &pl, const QueryTrack &qt) {
    cudaStream_t s = ctx->stream;
    CUDA_TRY(cudaEventRecord(ctx->kev[0], s));
    TRY(enqueue_select_plan(ctx, pl, qt, s));
    CUDA_TRY(cudaEventRecord(ctx->kev[1], s));
    TRY(enqueue_products(ctx, pl, qt, s));
    CUDA_TRY(cudaEventRecord(ctx->kev[2], s));
    CUDA_TRY(launch_advance_end(ctx->slots.as<MatSlot>(), (uint32_t)pl.slots.size(), pl.slot_rows, ctx->d_st, qt, 0, 0,
                                closure_counters(ctx, pl), s));
    CUDA_TRY(cudaEventRecord(ctx->kev[3], s));
    return CFPQ_OK;
}

static int accumulate_kernel_times(cfpq_ctx *ctx) {
    float t[3];
    for (int i = 0; i < 3; ++i) CUDA_TRY(cudaEventElapsedTime(&t[i], ctx->kev[i], ctx->kev[i + 1]));
    ctx->prof.plan_ms += t[0];
    ctx->prof.product_ms += t[1];
    ctx->prof.advance_ms += t[2];  // advance and iteration end are one kernel
    ctx->prof.plan_launches++;
    ctx->prof.product_launches++;
    ctx->prof.advance_launches++;
    return CFPQ_OK;
}

extern "C" int cfpq_calibrate(cfpq_ctx *ctx, cfpq_calibration *out) {
    TRY(use_device(ctx));
    if (!out) return set_error(CFPQ_ERR_INVALID, "null argument");
    memset(out, 0, sizeof(*out));
    TRY(ctx->stage.ensure((size_t)ctx->num_sms * 8 * 256 * 4));
    double ops = 0, ms = 0;
    CUDA_TRY(measure_logic_rate(ctx->num_sms, ctx->stage.as<uint32_t>(), ctx->stream, ctx->ev0, ctx->ev1, &ops, &ms));
    int clk_khz = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&clk_khz, cudaDevAttrClockRate, ctx->device));
    out->logic_ops_per_s = ops;
    out->logic_ops_per_clk_sm = clk_khz ? ops / ctx->num_sms / (clk_khz * 1e3) : 0;
    out->bitmac_per_s = 32.0 * ops;
    out->ms = ms;
    return CFPQ_OK;
}

extern "C" int cfpq_last_kernel_profile(cfpq_ctx *ctx, cfpq_kernel_profile *out) {
    if (!ctx || !out) return set_error(CFPQ_ERR_INVALID, "null argument");
    *out = ctx->prof;
    return CFPQ_OK;
}

// Build (or reuse) the CUDA graph: one while node whose body is one iteration.
static int get_loop_graph(cfpq_ctx *ctx, const ClosurePlan &pl, const QueryTrack &qt, cudaGraphExec_t *out) {
    std::vector<uint64_t> key = {(uint64_t)(uintptr_t)ctx->prods.p,  (uint64_t)pl.prods.size(),
                                 (uint64_t)pl.prod_rows,              (uint64_t)(uintptr_t)ctx->slots.p,
                                 (uint64_t)pl.slots.size(),           (uint64_t)pl.slot_rows,
                                 (uint64_t)(uintptr_t)ctx->items.p,   (uint64_t)(uintptr_t)ctx->prod_seen.p,
                                 (uint64_t)(uintptr_t)qt.changed,     (uint64_t)(uintptr_t)qt.last_iter,
                                 (uint64_t)(uintptr_t)qt.done_ns,     (uint64_t)ctx->lop3_grid,
                                 (uint64_t)pl.item_cap,               (uint64_t)(pl.uses_lop3 + 2 * pl.uses_m4r + 4 * pl.uses_tc),
                                 (uint64_t)(uintptr_t)ctx->choice.p,
                                 (uint64_t)(uintptr_t)ctx->cnts.p,    (uint64_t)(uintptr_t)ctx->d_sel.p,
                                 (uint64_t)(uintptr_t)ctx->tc_ok.p,   (uint64_t)(uintptr_t)ctx->sel_log.p,
                                 (uint64_t)ctx->sel_log_iters,        (uint64_t)pl.auto_select};
    key.push_back((uint64_t)(uintptr_t)ctx->tc_rows.p);  // the grouped tensor-core launches
    key.push_back(((uint64_t)pl.tc_rows.size() << 32) | pl.tc_groups);
    if (ctx->gcache.exec && ctx->gcache.key == key) {
        *out = ctx->gcache.exec;
        return CFPQ_OK;
    }
    ctx->gcache.release();
    cudaGraph_t graph = nullptr;
    CUDA_TRY(cudaGraphCreate(&graph, 0));
    cudaGraphConditionalHandle handle;
    CUDA_TRY(cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CUDA_TRY(cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CUDA_TRY(cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    int rc = enqueue_iteration(ctx, pl, qt, handle, 1);
    cudaGraph_t captured = nullptr;
    cudaError_t e = cudaStreamEndCapture(ctx->stream, &captured);
    if (rc != CFPQ_OK) {
        cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return set_error(CFPQ_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
    }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return set_error(CFPQ_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
    }
    ctx->gcache.graph = graph;
    ctx->gcache.exec = exec;
    ctx->gcache.key = key;
    *out = exec;
    return CFPQ_OK;
}

// Product records (features and the selector's decision, no timings) of the
// iterations the selection log holds.
static int collect_selection_log(cfpq_ctx *ctx, const ClosurePlan &pl, uint32_t iterations) {
    const uint32_t np = (uint32_t)pl.prods.size(), its = std::min(iterations, ctx->sel_log_iters);
    if (!np || !its) return CFPQ_OK;
    std::vector<SelLogRow> rows((size_t)its * np);
    CUDA_TRY(cudaMemcpy(rows.data(), ctx->sel_log.p, rows.size() * sizeof(SelLogRow), cudaMemcpyDeviceToHost));
    for (uint32_t it = 0; it < its; ++it)
        for (uint32_t p = 0; p < np; ++p) {
            const ProdDesc &pd = pl.prods[p];
            if (pd.term == 1 && it == 0) continue;  // the first iteration runs term 0 only
            const SelLogRow &r = rows[(size_t)it * np + p];
            cfpq_product_record rec;
            memset(&rec, 0, sizeof(rec));
            rec.iteration = it;
            rec.query = pd.query;
            rec.rule = pd.rule;
            rec.term = pd.term;
            rec.n = pd.n;
            rec.variant = r.choice & 0xFF;
            rec.flags = r.choice & ~0xFFu;
            memcpy(rec.features, r.f, sizeof(rec.features));
            memcpy(rec.predicted, r.pred, sizeof(rec.predicted));
            for (float &u : rec.usec) u = -1.f;
            ctx->log.push_back(rec);
        }
    return CFPQ_OK;
}

// CFPQ_LOG_PRODUCTS: iterations from the host.  Each iteration: the selector
// (features and decision of every term), the real work with the chosen
// variants, then every term alone with every candidate variant, timed with
// events (the state no longer changes: all bits are already there), then the
// iteration end.
static int run_logged_iterations(cfpq_ctx *ctx, const ClosurePlan &pl, const QueryTrack &qt) {
    cudaStream_t s = ctx->stream;
    const uint32_t np = (uint32_t)pl.prods.size();
    const int tpb = product_lop3_tiles_per_block();
    const size_t need_ev = (size_t)np * 3 * 2;
    while (ctx->tev.size() < need_ev) {
        cudaEvent_t e;
        CUDA_TRY(cudaEventCreate(&e));
        ctx->tev.push_back(e);
    }
    std::vector<int> tc_index(np, -1);
    for (size_t i = 0; i < pl.tc_prods.size(); ++i) tc_index[pl.tc_prods[i].index] = (int)i;
    std::vector<SelLogRow> rows(np);
    for (uint32_t it = 0;; ++it) {
        if (it > (1u << 20)) return set_error(CFPQ_ERR_CUDA, "closure did not converge");
        // features + decisions (always logged in this mode)
        CUDA_TRY(launch_select(ctx->prods.as<ProdDesc>(), np, ctx->cnts.as<BufCounters>(), ctx->d_st,
                               ctx->d_sel.as<SelectorParams>(), ctx->choice.as<uint8_t>(), ctx->tc_ok.as<uint8_t>(),
                               ctx->sel_log.as<SelLogRow>(), ctx->sel_log_iters, s));
        if (!pl.auto_select) CUDA_TRY(launch_fill_choice(ctx->choice.as<uint8_t>(), np, pl.fixed_variant, s));
        uint8_t *const kept = ctx->choice.as<uint8_t>() + np;
        CUDA_TRY(cudaMemcpyAsync(kept, ctx->choice.p, np, cudaMemcpyDeviceToDevice, s));
        // every term alone with every candidate variant, first, so that the
        // timings see the operands the selection saw (plus what the terms
        // timed before them added, as in a sequential pass); the candidates
        // are real products of this iteration: their new bits go to the
        // heads and the deltas like any other
        std::vector<std::pair<uint32_t, int>> timed;  // (product, variant)
        size_t ev = 0;
        for (uint32_t p = 0; p < np; ++p) {
            const ProdDesc &pd = pl.prods[p];
            if (pd.term == 1 && it == 0) continue;
            for (int v = CFPQ_VARIANT_LOP3; v <= CFPQ_VARIANT_TC; ++v) {
                if (v == CFPQ_VARIANT_TC && tc_index[p] < 0) continue;
                CUDA_TRY(cudaMemsetAsync(ctx->choice.as<uint8_t>() + p, v, 1, s));
                CUDA_TRY(cudaEventRecord(ctx->tev[ev], s));
                if (v == CFPQ_VARIANT_TC) {
                    TRY(launch_tc_product(ctx, pl.tc_prods[tc_index[p]], np, pl.item_cap, nullptr, qt.changed,
                                          ctx->choice.as<uint8_t>(), ctx->cnts.as<BufCounters>(), s));
                } else {
                    CUDA_TRY(launch_plan(ctx->prods.as<ProdDesc>(), np, pd.row_start, pd.row_start + pd.T,
                                         ctx->slots.as<MatSlot>(), ctx->d_st, ctx->items.as<uint64_t>(), pl.item_cap,
                                         tpb, nullptr, 0, ctx->choice.as<uint8_t>(), s));
                    TRY(launch_products(ctx, pl.item_cap, v == CFPQ_VARIANT_LOP3, v == CFPQ_VARIANT_M4R, qt.changed,
                                        ctx->cnts.as<BufCounters>(), s));
                    CUDA_TRY(launch_reset_list(ctx->d_st, v == CFPQ_VARIANT_LOP3 ? 0 : 1, s));
                }
                CUDA_TRY(cudaEventRecord(ctx->tev[ev + 1], s));
                ev += 2;
                timed.push_back({p, v});
            }
        }
        // then the iteration with the selector's choices (it finds little
        // new: the candidates did the same products)
        CUDA_TRY(cudaMemcpyAsync(ctx->choice.p, kept, np, cudaMemcpyDeviceToDevice, s));
        CUDA_TRY(launch_plan(ctx->prods.as<ProdDesc>(), np, 0, pl.prod_rows, ctx->slots.as<MatSlot>(), ctx->d_st,
                             ctx->items.as<uint64_t>(), pl.item_cap, tpb, ctx->prod_seen.as<uint32_t>(), 0,
                             ctx->choice.as<uint8_t>(), s));
        TRY(enqueue_products(ctx, pl, qt, s));
        CUDA_TRY(launch_reset_list(ctx->d_st, 0, s));
        CUDA_TRY(launch_reset_list(ctx->d_st, 1, s));
        CUDA_TRY(launch_advance_end(ctx->slots.as<MatSlot>(), (uint32_t)pl.slots.size(), pl.slot_rows, ctx->d_st, qt, 0,
                                    0, ctx->cnts.as<BufCounters>(), s));
        CUDA_TRY(cudaMemcpyAsync(ctx->h_st, ctx->d_st, sizeof(IterState), cudaMemcpyDeviceToHost, s));
        CUDA_TRY(cudaStreamSynchronize(s));
        if (it < ctx->sel_log_iters)
            CUDA_TRY(cudaMemcpy(rows.data(), ctx->sel_log.as<SelLogRow>() + (size_t)it * np, np * sizeof(SelLogRow),
                                cudaMemcpyDeviceToHost));
        std::vector<int> rec_of(np, -1);
        for (uint32_t p = 0; p < np; ++p) {
            const ProdDesc &pd = pl.prods[p];
            if (pd.term == 1 && it == 0) continue;
            cfpq_product_record rec;
            memset(&rec, 0, sizeof(rec));
            rec.iteration = it;
            rec.query = pd.query;
            rec.rule = pd.rule;
            rec.term = pd.term;
            rec.n = pd.n;
            const SelLogRow &r = rows[p];
            rec.variant = pl.auto_select ? (r.choice & 0xFF) : pl.fixed_variant;
            rec.flags = r.choice & ~0xFFu;
            memcpy(rec.features, r.f, sizeof(rec.features));
            memcpy(rec.predicted, r.pred, sizeof(rec.predicted));
            for (float &u : rec.usec) u = -1.f;
            rec_of[p] = (int)ctx->log.size();
            ctx->log.push_back(rec);
        }
        for (size_t i = 0; i < timed.size(); ++i) {
            float ms = 0;
            CUDA_TRY(cudaEventElapsedTime(&ms, ctx->tev[2 * i], ctx->tev[2 * i + 1]));
            ctx->log[rec_of[timed[i].first]].usec[timed[i].second] = ms * 1e3f;
        }
        if (!ctx->h_st->active) break;
    }
    return CFPQ_OK;
}

// Result lines wanted with a closure (cfpq_closure_hash): hashed on the
// device right after the closure, read back with the same synchronisation.
struct HashOut {
    cfpq_matrix *const *mats;
    size_t n;
    uint64_t *hashes, *counts;
    const uint32_t *flag_src;  // non-null: one device word read back with the same synchronisation
    uint32_t *flag_dst;        // (pinned host)
};

static void fill_hash_out(const cfpq_ctx *ctx, const HashOut *ho) {
    for (size_t i = 0; ho && i < ho->n; ++i) {
        ho->hashes[i] = ctx->h_hash[2 * i] % 1000000007ULL;
        ho->counts[i] = ctx->h_hash[2 * i + 1];
    }
}

static int run_engine(cfpq_ctx *ctx, const std::vector<QueryIn> &qs, const cfpq_closure_opts &o,
                      cfpq_closure_stats *stats, uint32_t *iters_out, double *done_ms_out,
                      const HashOut *ho = nullptr, const ClosureInput *input = nullptr) {
    for (size_t qi = 0; qi < qs.size(); ++qi) TRY(validate_query(qs[qi], qi));
    std::vector<uint64_t> key;
    plan_key(ctx, qs, o.variant, &key);
    if (!ctx->pcache) ctx->pcache = new PlanCache();
    PlanCache &pc = *ctx->pcache;
    if (!pc.valid || pc.key != key) {
        drop_plan_cache(ctx, false);
        int rc = build_plan(ctx, qs, o.variant, &pc.pl);
        if (rc != CFPQ_OK) {
            drop_plan_cache(ctx, false);
            return rc;
        }
        pc.valid = true;
        pc.key = std::move(key);
        pc.id = ++ctx->plan_ids;
    }
    ClosurePlan &pl = pc.pl;
    const size_t nq = qs.size();
    if (pl.prods.empty()) {
        if (input) CUDA_TRY(launch_closure_input(*input, ctx->num_sms, ctx->stream));  // sets input->bad to 0 first
        if (stats) memset(stats, 0, sizeof(*stats));
        for (size_t q = 0; q < nq; ++q) {
            if (iters_out) iters_out[q] = 0;
            if (done_ms_out) done_ms_out[q] = 0;
        }
        if (ho && ho->n) TRY(enqueue_hash_many(ctx, ho->mats, ho->n));
        if (ho && ho->flag_src)
            CUDA_TRY(cudaMemcpyAsync(ho->flag_dst, ho->flag_src, 4, cudaMemcpyDeviceToHost, ctx->stream));
        if (ho) {
            TRY(sync_and_check(ctx));
            fill_hash_out(ctx, ho);
        }
        return CFPQ_OK;
    }
    // device tables
    void *const slots_before = ctx->slots.p, *const prods_before = ctx->prods.p, *const qr_before = ctx->qranges.p;
    void *const tcok_before = ctx->tc_ok.p, *const tcr_before = ctx->tc_rows.p;
    TRY(ctx->slots.ensure(pl.slots.size() * sizeof(MatSlot)));
    TRY(ctx->prods.ensure(pl.prods.size() * sizeof(ProdDesc)));
    TRY(ctx->qranges.ensure(pl.qranges.size() * sizeof(QueryRange)));
    TRY(ctx->tc_ok.ensure(pl.prods.size()));
    TRY(ctx->tc_rows.ensure(pl.tc_rows.size() * sizeof(TcRows)));
    const bool tables_current = ctx->tables_owner == pc.id && ctx->slots.p == slots_before &&
                                ctx->prods.p == prods_before && ctx->qranges.p == qr_before &&
                                ctx->tc_ok.p == tcok_before && ctx->tc_rows.p == tcr_before;
    const bool timed = (o.log_products & CFPQ_LOG_KERNELS) != 0;
    const bool log_products = (o.log_products & CFPQ_LOG_PRODUCTS) != 0;
    const int persist_grid = ctx->persist_grid[pl.uses_m4r ? 1 : 0];
    const bool persistent =
        o.use_graph == CFPQ_LOOP_DEVICE && !timed && !log_products && !pl.uses_tc && persist_grid > 0;
    const uint32_t nprods = (uint32_t)pl.prods.size(), nslots = (uint32_t)pl.slots.size();
    TRY(ctx->items.ensure((persistent ? 4 : 3) * pl.item_cap * 8));
    // the persistent kernel's item lists: zero entries mean "not yet written";
    // a successful persistent closure leaves them zeroed (every item taken is
    // reset), so only other users of the buffer make a new zeroing necessary
    const size_t list_words = 3 * pl.item_cap * 2;
    const bool lists_clean = ctx->items_clean_ptr == ctx->items.p && ctx->items_clean_words >= list_words;
    ctx->items_clean_words = 0;
    TRY(ctx->choice.ensure(2 * (size_t)nprods));  // choices, then a copy kept by the product log
    TRY(ctx->cnts.ensure((size_t)nslots * 3 * sizeof(BufCounters)));
    ctx->cnts_on = pl.auto_select || log_products;
    if (ctx->cnts_on) TRY(selector_sync(ctx));
    ctx->sel_log_iters = (log_products || (o.log_products & CFPQ_LOG_SELECTION)) ? kSelLogIters : 0;
    ctx->sel_log_prods = nprods;
    if (ctx->sel_log_iters) TRY(ctx->sel_log.ensure((size_t)kSelLogIters * nprods * sizeof(SelLogRow)));
    ctx->log.clear();
    TRY(ctx->prod_seen.ensure(pl.prods.size() * 4));
    if (persistent) TRY(ctx->phase_log.ensure(kPhaseLogIters * 3 * 8));
    static_assert(sizeof(ItemTrace) == sizeof(cfpq_item_record), "item trace layout");
    const bool trace = persistent && (o.log_products & CFPQ_LOG_ITEMS) != 0;
    const size_t trace_bytes = (size_t)kItemTraceCap * sizeof(ItemTrace);
    ctx->item_trace_n = 0;
    if (trace) {
        TRY(ctx->item_trace.ensure(trace_bytes + 64));
        CUDA_TRY(cudaMemsetAsync(static_cast<char *>(ctx->item_trace.p) + trace_bytes, 0, 4, ctx->stream));
    }
    // done_ns, changed flags (three rotating arrays in the persistent kernel), last_iter
    const size_t qbytes = nq * (8 + 3 * 4 + 4) + 64;
    TRY(ctx->qtrack.ensure(qbytes));
    QueryTrack qt;
    qt.done_ns = ctx->qtrack.as<unsigned long long>();
    qt.changed = reinterpret_cast<uint32_t *>(qt.done_ns + nq);
    qt.last_iter = qt.changed + 3 * nq;
    if (!tables_current) {
        CUDA_TRY(cudaMemcpyAsync(ctx->slots.p, pl.slots.data(), pl.slots.size() * sizeof(MatSlot),
                                 cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(cudaMemcpyAsync(ctx->prods.p, pl.prods.data(), pl.prods.size() * sizeof(ProdDesc),
                                 cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(cudaMemcpyAsync(ctx->tc_ok.p, pl.tc_ok.data(), nprods, cudaMemcpyHostToDevice, ctx->stream));
        CUDA_TRY(cudaMemcpyAsync(ctx->qranges.p, pl.qranges.data(), pl.qranges.size() * sizeof(QueryRange),
                                 cudaMemcpyHostToDevice, ctx->stream));
        if (!pl.tc_rows.empty())
            CUDA_TRY(cudaMemcpyAsync(ctx->tc_rows.p, pl.tc_rows.data(), pl.tc_rows.size() * sizeof(TcRows),
                                     cudaMemcpyHostToDevice, ctx->stream));
        ctx->tables_owner = pc.id;
    }
    // the persistent kernel hands its final state (and the caller's flag
    // word, which lives in the pinned flag block) to the host itself
    const bool st_mapped = persistent && ctx->h_st_dev != nullptr;
    const bool flag_mapped = st_mapped && ho && ho->flag_src && ho->flag_dst >= ctx->h_flag &&
                             ho->flag_dst < ctx->h_flag + 16;
    // the closure prologue: product-seen flags, query tracking, the
    // persistent kernel's item lists (one per iteration parity, at 0 and 2 *
    // item_cap: a zero entry means "not yet written"), the variant choices and
    // the iteration state (zeroed, then active, limit, query count, start stamp)
    ClosureBegin b;
    memset(&b, 0, sizeof(b));
    b.zero[0] = ctx->prod_seen.as<uint32_t>();
    b.nwords[0] = pl.prods.size();
    b.zero[1] = ctx->qtrack.as<uint32_t>();
    b.nwords[1] = qbytes / 4;
    b.zero[2] = ctx->items.as<uint32_t>();
    b.nwords[2] = persistent && !lists_clean ? list_words : 0;
    b.choice = ctx->choice.as<uint8_t>();
    b.nchoice = nprods;
    b.choice_value = pl.auto_select ? (uint8_t)CFPQ_VARIANT_LOP3 : pl.fixed_variant;
    b.st = ctx->d_st;
    b.max_iter = o.max_iterations > 0 ? (uint32_t)o.max_iterations : 0;
    b.nqueries = (uint32_t)nq;
    // the query's input phase, enqueued right before the closure's own
    // launches (stand-alone kernels: as a prologue of the persistent kernel,
    // between two grid barriers, it measured ~10 us slower per query); its
    // first kernel clears the matrices and runs the closure prologue, which
    // touches neither the matrices nor the counters
    if (input) CUDA_TRY(launch_closure_input(*input, ctx->num_sms, ctx->stream, &b));
    if (ctx->cnts_on) CUDA_TRY(launch_counters_init(ctx->slots.as<MatSlot>(), nslots, ctx->cnts.as<BufCounters>(),
                                                    ctx->stream));
    if (ctx->sel_log_iters)
        CUDA_TRY(cudaMemsetAsync(ctx->sel_log.p, 0, (size_t)kSelLogIters * nprods * sizeof(SelLogRow), ctx->stream));
    if (!input) CUDA_TRY(launch_closure_begin(b, ctx->num_sms, ctx->stream));

    cudaGraphExec_t exec = nullptr;
    if (o.use_graph && !timed && !log_products && !persistent) TRY(get_loop_graph(ctx, pl, qt, &exec));
    if (timed) memset(&ctx->prof, 0, sizeof(ctx->prof));

    CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
    if (log_products) {
        TRY(run_logged_iterations(ctx, pl, qt));
    } else if (timed) {
        for (uint32_t it = 0;; ++it) {
            TRY(enqueue_iteration_timed(ctx, pl, qt));
            CUDA_TRY(cudaMemcpyAsync(ctx->h_st, ctx->d_st, sizeof(IterState), cudaMemcpyDeviceToHost, ctx->stream));
            CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            TRY(accumulate_kernel_times(ctx));
            if (!ctx->h_st->active) break;
            if (it > (1u << 24)) return set_error(CFPQ_ERR_CUDA, "closure did not converge");
        }
    } else if (persistent) {
        CUDA_TRY(launch_closure_persistent(pl.uses_m4r ? 1 : 0, persist_grid, ctx->prods.as<ProdDesc>(),
                                           (uint32_t)pl.prods.size(), pl.prod_rows, ctx->slots.as<MatSlot>(),
                                           (uint32_t)pl.slots.size(), pl.slot_rows, ctx->d_st,
                                           ctx->items.as<uint64_t>(), pl.item_cap, ctx->prod_seen.as<uint32_t>(), qt,
                                           product_lop3_tiles_per_block(),
                                           ctx->phase_log.as<unsigned long long>(), kPhaseLogIters,
                                           closure_counters(ctx, pl), ctx->choice.as<uint8_t>(),
                                           pl.auto_select ? ctx->d_sel.as<SelectorParams>() : nullptr,
                                           ctx->sel_log_iters ? ctx->sel_log.as<SelLogRow>() : nullptr,
                                           ctx->sel_log_iters,
                                           nq >= 2 && nq <= kMaxActiveQueries ? ctx->qranges.as<QueryRange>()
                                                                              : nullptr,
                                           trace ? ctx->item_trace.as<ItemTrace>() : nullptr,
                                           trace ? reinterpret_cast<uint32_t *>(
                                                       static_cast<char *>(ctx->item_trace.p) + trace_bytes)
                                                 : nullptr,
                                           // one small closure: latency-bound, merge without the read of C
                                           nq == 1 && pl.prods[0].T <= kDirectMergeMaxTiles ? 1 : 0,
                                           nq > 1 ? 1 : 0, (uint32_t)std::max(o.wait_limit, 0),
                                           (o.test_flags & CFPQ_TEST_STALL_BARRIER) != 0,
                                           st_mapped ? ctx->h_st_dev : nullptr,
                                           flag_mapped ? ho->flag_src : nullptr,
                                           flag_mapped ? ctx->h_flag_dev + (ho->flag_dst - ctx->h_flag) : nullptr,
                                           ctx->stream));
    } else if (exec) {
        CUDA_TRY(cudaGraphLaunch(exec, ctx->stream));
    } else {
        // Host loop: check the device flag every `batch` iterations; surplus
        // iterations after convergence are no-ops.
        const int batch = 4;
        uint32_t launched = 0;
        for (;;) {
            for (int k = 0; k < batch; ++k) TRY(enqueue_iteration(ctx, pl, qt, 0, 0));
            launched += batch;
            CUDA_TRY(cudaMemcpyAsync(ctx->h_st, ctx->d_st, sizeof(IterState), cudaMemcpyDeviceToHost, ctx->stream));
            CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            if (!ctx->h_st->active) break;
            if (launched > (1u << 24)) return set_error(CFPQ_ERR_CUDA, "closure did not converge");
        }
    }
    CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
    if (!st_mapped)
        CUDA_TRY(cudaMemcpyAsync(ctx->h_st, ctx->d_st, sizeof(IterState), cudaMemcpyDeviceToHost, ctx->stream));
    if (trace)
        CUDA_TRY(cudaMemcpyAsync(&ctx->item_trace_n, static_cast<char *>(ctx->item_trace.p) + trace_bytes, 4,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    // per-query results (only when asked for), through a pinned block
    const bool want_q = iters_out || done_ms_out;
    unsigned long long *h_done = nullptr;
    uint32_t *h_last = nullptr;
    if (want_q) {
        const size_t need = nq * 12;
        if (ctx->h_query_cap < need) {
            if (ctx->h_query) cudaFreeHost(ctx->h_query);
            ctx->h_query = nullptr;
            ctx->h_query_cap = 0;
            CUDA_TRY(cudaMallocHost(&ctx->h_query, need));
            ctx->h_query_cap = need;
        }
        h_done = static_cast<unsigned long long *>(ctx->h_query);
        h_last = reinterpret_cast<uint32_t *>(h_done + nq);
        CUDA_TRY(cudaMemcpyAsync(h_done, qt.done_ns, nq * 8, cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(cudaMemcpyAsync(h_last, qt.last_iter, nq * 4, cudaMemcpyDeviceToHost, ctx->stream));
    }
    if (ho && ho->n) TRY(enqueue_hash_many(ctx, ho->mats, ho->n));
    if (ho && ho->flag_src && !flag_mapped)
        CUDA_TRY(cudaMemcpyAsync(ho->flag_dst, ho->flag_src, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    const IterState &hs = *ctx->h_st;
    const bool converged = hs.last_changed == 0;
    ctx->phase_log_iters = persistent ? std::min<uint32_t>(hs.iter, kPhaseLogIters) : 0;
    if (hs.error) {
        drop_plan_cache(ctx, true);
        return set_error(CFPQ_ERR_TIMEOUT, "a bounded device wait gave up during the closure");
    }
    if (persistent) {
        ctx->items_clean_ptr = ctx->items.p;
        ctx->items_clean_words = list_words;
    }
    if (!converged)  // stopped by the iteration limit: the deltas still hold bits
        for (auto *m : pl.deltas) CUDA_TRY(launch_clear_matrix(m->d, ctx->stream));
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->iterations = hs.iter;
        stats->products = hs.products;
        stats->tile_triples = hs.tile_triples;
        stats->work_items = hs.items_total;
        stats->dense_bitops = hs.dense_bitops;
        stats->device_ms = ms;
        // the input phase (first kernel with the prologue, scatter, diagonals),
        // the counters, the prologue when it ran alone, the closure, the hash
        const uint64_t input_launches = input ? 1 + (input->nedges ? 1 : 0) + (input->ndiag ? 1 : 0) : 0;
        stats->kernel_launches = input_launches + (ctx->cnts_on ? 1 : 0) + (input ? 0 : 1) +
                                 (persistent ? 1 : (uint64_t)hs.iter * 3) +
                                 (ho && ho->n ? (ho->n + kHashBatch - 1) / kHashBatch : 0);
        stats->variant_items[CFPQ_VARIANT_LOP3] = hs.items_by_variant[2];
        stats->variant_items[CFPQ_VARIANT_M4R] = hs.items_by_variant[3];
        stats->variant_items[CFPQ_VARIANT_TC] = hs.items_by_variant[4];
        stats->bytes_staged = hs.bytes_staged;
        stats->out_words = hs.out_words;
        stats->new_words = hs.new_words;
    }
    for (size_t q = 0; want_q && q < nq; ++q) {
        if (iters_out) iters_out[q] = h_last[q];
        if (done_ms_out) done_ms_out[q] = h_last[q] ? (double)(h_done[q] - hs.t_start_ns) / 1e6 : 0.0;
    }
    if (ctx->sel_log_iters && !log_products) TRY(collect_selection_log(ctx, pl, hs.iter));
    fill_hash_out(ctx, ho);
    return CFPQ_OK;
}

static int run_worklist(cfpq_ctx *ctx, const QueryIn &q, const cfpq_closure_opts &o, cfpq_closure_stats *stats) {
    TRY(validate_query(q, 0));
    const size_t nr = q.nrules;
    std::vector<std::vector<uint32_t>> users(q.nmats);
    for (size_t r = 0; r < nr; ++r) {
        users[q.rules[r].body1].push_back((uint32_t)r);
        users[q.rules[r].body2].push_back((uint32_t)r);
    }
    std::deque<uint32_t> queue;
    std::vector<char> queued(nr, 1);
    for (size_t r = 0; r < nr; ++r) queue.push_back((uint32_t)r);
    const int variant = o.variant == CFPQ_VARIANT_AUTO ? CFPQ_VARIANT_LOP3 : o.variant;
    uint64_t products = 0;
    CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
    while (!queue.empty()) {
        const uint32_t r = queue.front();
        queue.pop_front();
        queued[r] = 0;
        const cfpq_rule &ru = q.rules[r];
        int changed = 0;
        TRY(cfpq_add_mul(ctx, q.mats[ru.head], q.mats[ru.body1], q.mats[ru.body2], variant, &changed));
        ++products;
        if (changed) {
            for (uint32_t u : users[ru.head])
                if (!queued[u]) {
                    queued[u] = 1;
                    queue.push_back(u);
                }
        }
        if (o.max_iterations > 0 && products >= (uint64_t)o.max_iterations) break;
    }
    CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
    CUDA_TRY(cudaEventSynchronize(ctx->ev1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->products = products;
        const uint64_t n = q.nmats ? q.mats[0]->d.n : 0;
        stats->dense_bitops = products * n * n * n;
        stats->device_ms = ms;
        stats->kernel_launches = products;
    }
    return CFPQ_OK;
}

// Variant NTSET: pack the query's matrices into one matrix of nonterminal
// sets, square it on the device until a pass changes nothing (the changed
// flag read back after each pass: the number of passes grows with the
// logarithm of the longest derivation), unpack into the matrices.
static int run_ntset(cfpq_ctx *ctx, const QueryIn &q, const cfpq_closure_opts &o, cfpq_closure_stats *stats) {
    TRY(validate_query(q, 0));
    if (stats) memset(stats, 0, sizeof(*stats));
    if (q.nmats > 32)
        return set_error(CFPQ_ERR_UNSUPPORTED, "nonterminal-set variant: %zu nonterminals (at most 32)", q.nmats);
    const uint32_t nm = (uint32_t)q.nmats;
    const uint32_t n = nm ? q.mats[0]->d.n : 0;
    if (n > ntset_max_n(nm))
        return set_error(CFPQ_ERR_UNSUPPORTED, "nonterminal-set variant: n = %u above %zu for %u nonterminals", n,
                         ntset_max_n(nm), nm);
    if (!n || !q.nrules) return CFPQ_OK;
    const uint32_t stride = q.mats[0]->d.T * 64;
    const size_t cb = ntset_cell_bytes(nm);
    TRY(ctx->nt_cells.ensure((size_t)stride * stride * cb));
    TRY(ctx->nt_mats.ensure(nm * sizeof(DevMat)));
    TRY(ctx->nt_rules.ensure(q.nrules * 4));
    TRY(ctx->nt_ctr.ensure(8));
    std::vector<DevMat> dm(nm);
    for (uint32_t i = 0; i < nm; ++i) dm[i] = q.mats[i]->d;
    std::vector<uint8_t> rules(q.nrules * 4);
    uint32_t ymask = 0;
    for (size_t r = 0; r < q.nrules; ++r) {
        rules[4 * r] = (uint8_t)q.rules[r].head;
        rules[4 * r + 1] = (uint8_t)q.rules[r].body1;
        rules[4 * r + 2] = (uint8_t)q.rules[r].body2;
        rules[4 * r + 3] = 0;
        ymask |= 1u << q.rules[r].body1;
    }
    ctx->tables_owner = 0;
    CUDA_TRY(cudaMemcpyAsync(ctx->nt_mats.p, dm.data(), nm * sizeof(DevMat), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(ctx->nt_rules.p, rules.data(), rules.size(), cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaEventRecord(ctx->ev0, ctx->stream));
    CUDA_TRY(launch_ntset_pack(ctx->nt_cells.p, stride, nm, ctx->nt_mats.as<DevMat>(), ctx->num_sms, ctx->stream));
    uint32_t passes = 0;
    for (;;) {
        CUDA_TRY(cudaMemsetAsync(ctx->nt_ctr.p, 0, 8, ctx->stream));
        CUDA_TRY(launch_ntset_square(ctx->nt_cells.p, n, stride, nm, ctx->nt_rules.p, (uint32_t)q.nrules, ymask,
                                     ctx->nt_ctr.as<uint32_t>(), ctx->num_sms, ctx->stream));
        ++passes;
        CUDA_TRY(cudaMemcpyAsync(ctx->h_flag, ctx->nt_ctr.as<uint32_t>() + 1, 4, cudaMemcpyDeviceToHost, ctx->stream));
        CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (!ctx->h_flag[0]) break;
        if (o.max_iterations > 0 && passes >= (uint32_t)o.max_iterations) break;
    }
    CUDA_TRY(launch_ntset_unpack(ctx->nt_cells.p, stride, nm, ctx->nt_mats.as<DevMat>(), ctx->num_sms, ctx->stream));
    for (uint32_t i = 0; i < nm; ++i) CUDA_TRY(launch_occ_rebuild(q.mats[i]->d, ctx->stream));
    CUDA_TRY(cudaEventRecord(ctx->ev1, ctx->stream));
    CUDA_TRY(cudaEventSynchronize(ctx->ev1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    if (stats) {
        stats->iterations = passes;
        stats->products = passes;
        stats->dense_bitops = (uint64_t)passes * n * n * n;
        stats->device_ms = ms;
        stats->kernel_launches = 2 + (uint64_t)passes + nm;
    }
    return CFPQ_OK;
}

static cfpq_closure_opts default_opts() {
    cfpq_closure_opts o;
    memset(&o, 0, sizeof(o));
    o.driver = CFPQ_DRIVER_ENGINE;
    o.variant = CFPQ_VARIANT_AUTO;
    o.use_graph = 1;
    return o;
}

extern "C" int cfpq_closure(cfpq_ctx *ctx, const cfpq_rule *rules, size_t nrules, cfpq_matrix *const *mats,
                            size_t nmats, const cfpq_closure_opts *opts, cfpq_closure_stats *stats) {
    TRY(use_device(ctx));
    const cfpq_closure_opts o = opts ? *opts : default_opts();
    QueryIn q{rules, nrules, mats, nmats};
    if (o.driver == CFPQ_DRIVER_WORKLIST) return run_worklist(ctx, q, o, stats);
    if (o.driver != CFPQ_DRIVER_ENGINE) return set_error(CFPQ_ERR_INVALID, "unknown driver %d", o.driver);
    if (o.variant == CFPQ_VARIANT_NTSET) return run_ntset(ctx, q, o, stats);
    if (o.variant == CFPQ_VARIANT_TC && !ctx->tc_grid)
        return set_error(CFPQ_ERR_UNSUPPORTED, "tensor-core variant unavailable (needs one CTA per SM)");
    if (o.variant != CFPQ_VARIANT_AUTO && o.variant != CFPQ_VARIANT_LOP3 && o.variant != CFPQ_VARIANT_M4R &&
        o.variant != CFPQ_VARIANT_TC)
        return set_error(CFPQ_ERR_UNSUPPORTED, "variant %d is not available in the engine driver", o.variant);
    std::vector<QueryIn> qs{q};
    return run_engine(ctx, qs, o, stats, nullptr, nullptr);
}

extern "C" int cfpq_closure_hash(cfpq_ctx *ctx, const cfpq_rule *rules, size_t nrules, cfpq_matrix *const *mats,
                                 size_t nmats, const cfpq_closure_opts *opts, cfpq_closure_stats *stats,
                                 uint64_t *hashes, uint64_t *counts) {
    TRY(use_device(ctx));
    if (nmats && (!hashes || !counts)) return set_error(CFPQ_ERR_INVALID, "null result array");
    const cfpq_closure_opts o = opts ? *opts : default_opts();
    if (o.driver != CFPQ_DRIVER_ENGINE || o.variant == CFPQ_VARIANT_NTSET) {
        TRY(cfpq_closure(ctx, rules, nrules, mats, nmats, opts, stats));
        return cfpq_hash_count_many(ctx, mats, nmats, hashes, counts);
    }
    if (o.variant == CFPQ_VARIANT_TC && !ctx->tc_grid)
        return set_error(CFPQ_ERR_UNSUPPORTED, "tensor-core variant unavailable (needs one CTA per SM)");
    if (o.variant != CFPQ_VARIANT_AUTO && o.variant != CFPQ_VARIANT_LOP3 && o.variant != CFPQ_VARIANT_M4R &&
        o.variant != CFPQ_VARIANT_TC)
        return set_error(CFPQ_ERR_UNSUPPORTED, "variant %d is not available in the engine driver", o.variant);
    std::vector<QueryIn> qs{QueryIn{rules, nrules, mats, nmats}};
    HashOut ho{mats, nmats, hashes, counts, nullptr, nullptr};
    return run_engine(ctx, qs, o, stats, nullptr, nullptr, &ho);
}

// The epsilon matrices' descriptors on the device, re-sent only when they
// differ from the last call's.
static int prepare_diag(cfpq_ctx *ctx, cfpq_matrix *const *mats, const uint32_t *epsilon, size_t nepsilon,
                        ClosureInput *in) {
    in->ndiag = 0;
    if (!nepsilon) return CFPQ_OK;
    std::vector<DevMat> tab(nepsilon);
    for (size_t i = 0; i < nepsilon; ++i) tab[i] = mats[epsilon[i]]->d;
    void *const before = ctx->diag_desc.p;
    TRY(ctx->diag_desc.ensure(nepsilon * sizeof(DevMat)));
    const unsigned char *tb = reinterpret_cast<const unsigned char *>(tab.data());
    std::vector<unsigned char> key(tb, tb + nepsilon * sizeof(DevMat));
    if (ctx->diag_desc.p != before || key != ctx->diag_desc_key) {
        ctx->diag_desc_key.clear();
        // synchronous: the descriptors are small and change only with the query
        CUDA_TRY(cudaMemcpy(ctx->diag_desc.p, tab.data(), nepsilon * sizeof(DevMat), cudaMemcpyHostToDevice));
        ctx->diag_desc_key = std::move(key);
    }
    in->diag = ctx->diag_desc.as<DevMat>();
    in->ndiag = (uint32_t)nepsilon;
    return CFPQ_OK;
}

// Slot of the context's pinned flag block that receives the edge scatter's
// out-of-range count in cfpq_intersection (slot 0 belongs to the
// synchronous flag reads).
constexpr int kIntersectBadSlot = 8;

static int intersection_impl(cfpq_ctx *ctx, const cfpq_rule *rules, size_t nrules, cfpq_matrix *const *mats,
                             size_t nmats, const cfpq_edges *edges, const uint32_t *epsilon, size_t nepsilon,
                             const cfpq_closure_opts *opts, cfpq_closure_stats *stats, uint64_t *hashes,
                             uint64_t *counts, bool *read_in_place) {
    if (!edges) return set_error(CFPQ_ERR_INVALID, "null edge list");
    if (nepsilon && !epsilon) return set_error(CFPQ_ERR_INVALID, "null epsilon list");
    if (nmats && !mats) return set_error(CFPQ_ERR_INVALID, "null matrix list");
    for (size_t i = 0; i < nmats; ++i)
        if (!mats[i]) return set_error(CFPQ_ERR_INVALID, "matrix %zu is null", i);
    const bool want_lines = hashes != nullptr || counts != nullptr;
    if (want_lines && (!hashes || !counts)) return set_error(CFPQ_ERR_INVALID, "hashes and counts go together");
    for (size_t i = 0; i < nepsilon; ++i)
        if (epsilon[i] >= nmats)
            return set_error(CFPQ_ERR_INVALID, "epsilon[%zu] = %u is not a matrix of the query", i, epsilon[i]);
    const cfpq_closure_opts o = opts ? *opts : default_opts();
    // the input phase: clear, scatter, diagonals
    ClosureInput in;
    memset(&in, 0, sizeof(in));
    TRY(prepare_clear(ctx, mats, nmats, &in));
    // the call returns only after its final synchronisation, so pinned host
    // edges can be read in place by the scatter kernel
    TRY(prepare_edges(ctx, mats, nmats, edges->from, edges->label, edges->to, edges->count, edges->label_offsets,
                      edges->label_mats, edges->nlabels, edges->on_device != 0, &in, true, read_in_place));
    TRY(prepare_diag(ctx, mats, epsilon, nepsilon, &in));
    in.bad = in.nedges ? ctx->d_bad : nullptr;
    uint32_t *const h_bad = ctx->h_flag + kIntersectBadSlot;
    *h_bad = 0;
    const bool engine = o.driver == CFPQ_DRIVER_ENGINE &&
                        (o.variant == CFPQ_VARIANT_AUTO || o.variant == CFPQ_VARIANT_LOP3 ||
                         o.variant == CFPQ_VARIANT_M4R || (o.variant == CFPQ_VARIANT_TC && ctx->tc_grid));
    if (engine) {
        // the engine runs the input phase itself (in the persistent kernel's
        // prologue when it can) and reads the scatter's count back with its
        // own final read-back: one synchronisation in all
        std::vector<QueryIn> qs{QueryIn{rules, nrules, mats, nmats}};
        HashOut ho{mats, want_lines ? nmats : 0, hashes, counts, in.bad, h_bad};
        TRY(run_engine(ctx, qs, o, stats, nullptr, nullptr, &ho, &in));
    } else {
        CUDA_TRY(launch_closure_input(in, ctx->num_sms, ctx->stream));  // sets in.bad to 0 first
        if (in.bad) CUDA_TRY(cudaMemcpyAsync(h_bad, in.bad, 4, cudaMemcpyDeviceToHost, ctx->stream));
        TRY(cfpq_closure(ctx, rules, nrules, mats, nmats, &o, stats));
        if (want_lines) TRY(cfpq_hash_count_many(ctx, mats, nmats, hashes, counts));
        else TRY(sync_and_check(ctx));
    }
    if (*h_bad) return set_error(CFPQ_ERR_INVALID, "cfpq_intersection: %u edge coordinates out of range", *h_bad);
    return CFPQ_OK;
}

extern "C" int cfpq_intersection(cfpq_ctx *ctx, const cfpq_rule *rules, size_t nrules, cfpq_matrix *const *mats,
                                 size_t nmats, const cfpq_edges *edges, const uint32_t *epsilon, size_t nepsilon,
                                 const cfpq_closure_opts *opts, cfpq_closure_stats *stats, uint64_t *hashes,
                                 uint64_t *counts) {
    TRY(use_device(ctx));
    bool in_place = false;
    const int rc = intersection_impl(ctx, rules, nrules, mats, nmats, edges, epsilon, nepsilon, opts, stats, hashes,
                                     counts, &in_place);
    // the scatter read the caller's pinned edges in place: never return
    // while it may still run (the error paths skip the final synchronisation)
    if (rc != CFPQ_OK && in_place) cudaStreamSynchronize(ctx->stream);
    return rc;
}

extern "C" int cfpq_closure_batch(cfpq_ctx *ctx, const cfpq_query *queries, size_t nqueries,
                                  const cfpq_closure_opts *opts, cfpq_closure_stats *stats, uint32_t *iterations_out,
                                  double *done_ms_out) {
    TRY(use_device(ctx));
    if (nqueries && !queries) return set_error(CFPQ_ERR_INVALID, "null query array");
    const cfpq_closure_opts o = opts ? *opts : default_opts();
    if (o.driver != CFPQ_DRIVER_ENGINE) return set_error(CFPQ_ERR_INVALID, "batched closure needs the engine driver");
    if (o.variant == CFPQ_VARIANT_TC && !ctx->tc_grid)
        return set_error(CFPQ_ERR_UNSUPPORTED, "tensor-core variant unavailable (needs one CTA per SM)");
    if (o.variant != CFPQ_VARIANT_AUTO && o.variant != CFPQ_VARIANT_LOP3 && o.variant != CFPQ_VARIANT_M4R &&
        o.variant != CFPQ_VARIANT_TC)
        return set_error(CFPQ_ERR_UNSUPPORTED, "variant %d is not available in the engine driver", o.variant);
    std::vector<QueryIn> qs;
    qs.reserve(nqueries);
    for (size_t i = 0; i < nqueries; ++i) qs.push_back({queries[i].rules, queries[i].nrules, queries[i].mats, queries[i].nmats});
    return run_engine(ctx, qs, o, stats, iterations_out, done_ms_out);
}

extern "C" size_t cfpq_last_phase_log(cfpq_ctx *ctx, uint64_t *out, size_t cap) {
    if (!ctx) return 0;
    const size_t n = ctx->phase_log_iters;
    const size_t k = std::min(cap, 3 * n);
    if (out && k) {
        if (cudaMemcpy(out, ctx->phase_log.p, k * 8, cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
    }
    return n;
}

extern "C" size_t cfpq_item_log(cfpq_ctx *ctx, cfpq_item_record *out, size_t cap) {
    if (!ctx) return 0;
    const size_t n = std::min<size_t>(ctx->item_trace_n, kItemTraceCap);
    const size_t k = std::min(cap, n);
    if (out && k && cudaMemcpy(out, ctx->item_trace.p, k * sizeof(cfpq_item_record), cudaMemcpyDeviceToHost) !=
                        cudaSuccess)
        return 0;
    return n;
}

extern "C" size_t cfpq_product_log(cfpq_ctx *ctx, cfpq_product_record *out, size_t cap) {
    if (!ctx) return 0;
    const size_t n = ctx->log.size();
    if (out) memcpy(out, ctx->log.data(), std::min(n, cap) * sizeof(cfpq_product_record));
    return n;
}
