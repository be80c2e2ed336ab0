// C ABI of the variant selector: configuration, cost-model weights, training
// on the GPU, the gradient-check and prediction entry points, and the
// autotuner that sets the heuristic's thresholds.  Declared in cfpq_b200.h.
#include <chrono>
#include <cmath>

#include "ctx.h"

void selector_defaults(SelectorParams *sp) {
    memset(sp, 0, sizeof(*sp));
    sp->mode = CFPQ_SELECT_HEURISTIC;
    sp->allowed = (1u << CFPQ_VARIANT_LOP3) | (1u << CFPQ_VARIANT_M4R) | (1u << CFPQ_VARIANT_TC);
    // Until cfpq_autotune runs: tensor cores for n >= 2048 when a fifth of
    // the P tiles are occupied and 30% of them dense (fit to the exhaustive
    // per-term timings of a chain closure at n = 32768; n >= 2048 from the
    // 512-query batch, whose tensor-core terms of all queries share one plan
    // and one product launch per iteration: 1.59 s without them, 1.18 s from
    // n = 4096, 1.13 s from n = 2048); Four Russians when a quarter of the P
    // tiles are dense.  (A single query selects only from n >= 64 *
    // min_tiles.)
    sp->tc_min_tiles = 32;
    sp->tc_min_occ = 0.2f;
    sp->tc_min_dense = 0.3f;
    sp->m4r_min_dense = 0.25f;
    sp->conf_margin = 0.05f;
    sp->range_margin = 0.1f;
    // Per-iteration selection costs one feature computation per planned row
    // and exact buffer counters in every epilogue; a single same-generation
    // query at n = 8192 (T = 128) loses 16% to it, with nothing to gain.
    // Batches of queries always select (512 mixed queries: 6-10% faster).
    sp->min_tiles = 256;
}

int selector_sync(cfpq_ctx *ctx) {
    if (!ctx->sel_dirty && ctx->d_sel.p) return CFPQ_OK;
    TRY(ctx->d_sel.ensure(sizeof(SelectorParams)));
    CUDA_TRY(cudaMemcpyAsync(ctx->d_sel.p, &ctx->sel, sizeof(SelectorParams), cudaMemcpyHostToDevice, ctx->stream));
    ctx->sel_dirty = false;
    return CFPQ_OK;
}

static int use_ctx(cfpq_ctx *ctx) {
    if (!ctx) return set_error(CFPQ_ERR_INVALID, "null context");
    CUDA_TRY(cudaSetDevice(ctx->device));
    return CFPQ_OK;
}

extern "C" int cfpq_selector_configure(cfpq_ctx *ctx, const cfpq_selector_config *cfg) {
    TRY(use_ctx(ctx));
    if (!cfg) return set_error(CFPQ_ERR_INVALID, "null configuration");
    if (cfg->mode < CFPQ_SELECT_FIXED || cfg->mode > CFPQ_SELECT_MLP)
        return set_error(CFPQ_ERR_INVALID, "unknown selector mode %d", cfg->mode);
    const uint32_t word = (1u << CFPQ_VARIANT_LOP3) | (1u << CFPQ_VARIANT_M4R);
    if ((cfg->allowed & ~(word | (1u << CFPQ_VARIANT_TC))) || !(cfg->allowed & word))
        return set_error(CFPQ_ERR_INVALID, "allowed variants 0x%x: only LOP3, M4R, TC, and at least one of LOP3/M4R",
                         cfg->allowed);
    if (cfg->mode == CFPQ_SELECT_MLP && !ctx->sel.has_weights)
        return set_error(CFPQ_ERR_INVALID, "MLP mode needs weights (cfpq_selector_train or cfpq_selector_set_weights)");
    SelectorParams &sp = ctx->sel;
    sp.mode = cfg->mode;
    sp.allowed = cfg->allowed & (ctx->tc_grid ? ~0u : ~(1u << CFPQ_VARIANT_TC));
    sp.tc_min_tiles = std::max<uint32_t>(cfg->tc_min_tiles, 1);
    sp.tc_min_occ = cfg->tc_min_occ;
    sp.tc_min_dense = cfg->tc_min_dense;
    sp.m4r_min_dense = cfg->m4r_min_dense;
    sp.conf_margin = cfg->conf_margin;
    sp.range_margin = cfg->range_margin;
    sp.min_tiles = cfg->min_tiles;
    ctx->sel_dirty = true;
    return CFPQ_OK;
}

extern "C" int cfpq_selector_get_config(cfpq_ctx *ctx, cfpq_selector_config *cfg) {
    if (!ctx || !cfg) return set_error(CFPQ_ERR_INVALID, "null argument");
    const SelectorParams &sp = ctx->sel;
    cfg->mode = sp.mode;
    cfg->allowed = sp.allowed;
    cfg->tc_min_tiles = sp.tc_min_tiles;
    cfg->tc_min_occ = sp.tc_min_occ;
    cfg->tc_min_dense = sp.tc_min_dense;
    cfg->m4r_min_dense = sp.m4r_min_dense;
    cfg->conf_margin = sp.conf_margin;
    cfg->range_margin = sp.range_margin;
    cfg->min_tiles = sp.min_tiles;
    return CFPQ_OK;
}

extern "C" size_t cfpq_selector_weight_count(void) { return (size_t)kSelWeights + 2 * kSelFeatures; }

extern "C" int cfpq_selector_set_weights(cfpq_ctx *ctx, const float *w, size_t count) {
    if (!ctx || !w) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (count != cfpq_selector_weight_count())
        return set_error(CFPQ_ERR_INVALID, "expected %zu floats, got %zu", cfpq_selector_weight_count(), count);
    for (size_t i = 0; i < count; ++i)
        if (!std::isfinite(w[i])) return set_error(CFPQ_ERR_INVALID, "weight %zu is not finite", i);
    memcpy(ctx->sel.w, w, sizeof(float) * kSelWeights);
    memcpy(ctx->sel.feat_lo, w + kSelWeights, sizeof(float) * kSelFeatures);
    memcpy(ctx->sel.feat_hi, w + kSelWeights + kSelFeatures, sizeof(float) * kSelFeatures);
    ctx->sel.has_weights = 1;
    ctx->sel_dirty = true;
    return CFPQ_OK;
}

extern "C" int cfpq_selector_get_weights(cfpq_ctx *ctx, float *w, size_t count) {
    if (!ctx || !w) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (!ctx->sel.has_weights) return set_error(CFPQ_ERR_INVALID, "the cost model has no weights yet");
    if (count < cfpq_selector_weight_count())
        return set_error(CFPQ_ERR_INVALID, "need %zu floats", cfpq_selector_weight_count());
    memcpy(w, ctx->sel.w, sizeof(float) * kSelWeights);
    memcpy(w + kSelWeights, ctx->sel.feat_lo, sizeof(float) * kSelFeatures);
    memcpy(w + kSelWeights + kSelFeatures, ctx->sel.feat_hi, sizeof(float) * kSelFeatures);
    return CFPQ_OK;
}

// Upload samples x[n][F], y[n][O], m[n][O] into the context's training buffers.
static int upload_samples(cfpq_ctx *ctx, const float *x, const float *y, const float *m, size_t n) {
    TRY(ctx->mlp_x.ensure(n * kSelFeatures * 4));
    TRY(ctx->mlp_y.ensure(n * kSelOutputs * 4));
    TRY(ctx->mlp_m.ensure(n * kSelOutputs * 4));
    CUDA_TRY(cudaMemcpyAsync(ctx->mlp_x.p, x, n * kSelFeatures * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (y) CUDA_TRY(cudaMemcpyAsync(ctx->mlp_y.p, y, n * kSelOutputs * 4, cudaMemcpyHostToDevice, ctx->stream));
    if (m) CUDA_TRY(cudaMemcpyAsync(ctx->mlp_m.p, m, n * kSelOutputs * 4, cudaMemcpyHostToDevice, ctx->stream));
    return CFPQ_OK;
}

static int ensure_train_state(cfpq_ctx *ctx) {
    TRY(ctx->mlp_w.ensure(kSelWeights * 4));
    TRY(ctx->mlp_grad.ensure(kSelWeights * 4));
    TRY(ctx->mlp_m1.ensure(kSelWeights * 4));
    TRY(ctx->mlp_v2.ensure(kSelWeights * 4));
    TRY(ctx->mlp_loss.ensure(64));
    return CFPQ_OK;
}

extern "C" int cfpq_selector_loss_grad(cfpq_ctx *ctx, const float *weights, const float *x, const float *y,
                                       const float *m, size_t n, float *loss, float *grad) {
    TRY(use_ctx(ctx));
    if (!weights || !x || !y || !m || !loss || !grad) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (n == 0 || n > (1u << 24)) return set_error(CFPQ_ERR_INVALID, "sample count %zu out of range", n);
    double msum = 0;
    for (size_t i = 0; i < n * kSelOutputs; ++i) msum += m[i];
    if (msum <= 0) return set_error(CFPQ_ERR_INVALID, "empty mask");
    TRY(ensure_train_state(ctx));
    TRY(upload_samples(ctx, x, y, m, n));
    CUDA_TRY(cudaMemcpyAsync(ctx->mlp_w.p, weights, kSelWeights * 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemsetAsync(ctx->mlp_grad.p, 0, kSelWeights * 4, ctx->stream));
    CUDA_TRY(cudaMemsetAsync(ctx->mlp_loss.p, 0, 4, ctx->stream));
    CUDA_TRY(mlp_loss_grad(ctx->mlp_w.as<float>(), ctx->mlp_x.as<float>(), ctx->mlp_y.as<float>(),
                           ctx->mlp_m.as<float>(), (uint32_t)n, (float)(1.0 / msum), ctx->mlp_grad.as<float>(),
                           ctx->mlp_loss.as<float>(), ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(grad, ctx->mlp_grad.p, kSelWeights * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(loss, ctx->mlp_loss.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return CFPQ_OK;
}

extern "C" int cfpq_selector_predict(cfpq_ctx *ctx, const float *x, size_t n, float *out) {
    TRY(use_ctx(ctx));
    if (!x || !out) return set_error(CFPQ_ERR_INVALID, "null argument");
    if (!ctx->sel.has_weights) return set_error(CFPQ_ERR_INVALID, "the cost model has no weights yet");
    if (n == 0) return CFPQ_OK;
    if (n > (1u << 24)) return set_error(CFPQ_ERR_INVALID, "sample count %zu out of range", n);
    TRY(ensure_train_state(ctx));
    TRY(upload_samples(ctx, x, nullptr, nullptr, n));
    TRY(ctx->mlp_out.ensure(n * kSelOutputs * 4));
    CUDA_TRY(cudaMemcpyAsync(ctx->mlp_w.p, ctx->sel.w, kSelWeights * 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(mlp_predict(ctx->mlp_w.as<float>(), ctx->mlp_x.as<float>(), (uint32_t)n, ctx->mlp_out.as<float>(),
                         ctx->stream));
    CUDA_TRY(cudaMemcpyAsync(out, ctx->mlp_out.p, n * kSelOutputs * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return CFPQ_OK;
}

// splitmix64 stream for the weight initialisation
static uint64_t mix64(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

extern "C" int cfpq_selector_train(cfpq_ctx *ctx, const cfpq_product_record *recs, size_t count,
                                   const cfpq_train_opts *opts, cfpq_train_report *report) {
    TRY(use_ctx(ctx));
    if (!recs && count) return set_error(CFPQ_ERR_INVALID, "null records");
    cfpq_train_opts o = {2000, 3e-3f, 1e-4f, 1, 0};
    if (opts) o = *opts;
    if (o.epochs <= 0 || o.epochs > 1000000) return set_error(CFPQ_ERR_INVALID, "epochs %d out of range", o.epochs);
    // samples: records with at least one timed candidate variant
    std::vector<float> X, Y, M;
    double ysum[kSelOutputs] = {0, 0, 0}, ycnt[kSelOutputs] = {0, 0, 0};
    for (size_t i = 0; i < count; ++i) {
        const cfpq_product_record &r = recs[i];
        float y[kSelOutputs], m[kSelOutputs];
        bool any = false;
        for (int j = 0; j < kSelOutputs; ++j) {
            const float us = r.usec[CFPQ_VARIANT_LOP3 + j];
            m[j] = us > 0.f ? 1.f : 0.f;
            y[j] = us > 0.f ? logf(us) : 0.f;
            if (us > 0.f) {
                any = true;
                ysum[j] += y[j];
                ycnt[j] += 1;
            }
        }
        if (!any) continue;
        X.insert(X.end(), r.features, r.features + kSelFeatures);
        Y.insert(Y.end(), y, y + kSelOutputs);
        M.insert(M.end(), m, m + kSelOutputs);
    }
    const size_t n = M.size() / kSelOutputs;
    if (n == 0) return set_error(CFPQ_ERR_INVALID, "no record has a timed variant (use CFPQ_LOG_PRODUCTS)");
    double msum = 0;
    for (float v : M) msum += v;
    // feature range of the training set
    SelectorParams &sp = ctx->sel;
    for (int f = 0; f < kSelFeatures; ++f) {
        float lo = X[f], hi = X[f];
        for (size_t i = 1; i < n; ++i) {
            lo = std::min(lo, X[i * kSelFeatures + f]);
            hi = std::max(hi, X[i * kSelFeatures + f]);
        }
        sp.feat_lo[f] = lo;
        sp.feat_hi[f] = hi;
    }
    if (!(o.keep_weights && sp.has_weights)) {  // Glorot-uniform layers, output bias = mean log time
        uint64_t st = 0x5DEECE66DULL ^ ((uint64_t)o.seed << 17);
        auto fill = [&](float *w, int fan_in, int fan_out, int cnt) {
            const float a = sqrtf(6.f / (float)(fan_in + fan_out));
            for (int i = 0; i < cnt; ++i) w[i] = a * (2.f * (float)((mix64(st) >> 40) * (1.0 / 16777216.0)) - 1.f);
        };
        float *w = sp.w;
        fill(w, kSelFeatures, kSelHidden, kSelFeatures * kSelHidden);
        w += kSelFeatures * kSelHidden;
        for (int i = 0; i < kSelHidden; ++i) *w++ = 0.f;
        fill(w, kSelHidden, kSelHidden, kSelHidden * kSelHidden);
        w += kSelHidden * kSelHidden;
        for (int i = 0; i < kSelHidden; ++i) *w++ = 0.f;
        fill(w, kSelHidden, kSelOutputs, kSelHidden * kSelOutputs);
        w += kSelHidden * kSelOutputs;
        for (int j = 0; j < kSelOutputs; ++j) *w++ = ycnt[j] > 0 ? (float)(ysum[j] / ycnt[j]) : 0.f;
    }
    TRY(ensure_train_state(ctx));
    TRY(upload_samples(ctx, X.data(), Y.data(), M.data(), n));
    CUDA_TRY(cudaMemcpyAsync(ctx->mlp_w.p, sp.w, kSelWeights * 4, cudaMemcpyHostToDevice, ctx->stream));
    CUDA_TRY(cudaMemsetAsync(ctx->mlp_grad.p, 0, kSelWeights * 4, ctx->stream));
    CUDA_TRY(cudaMemsetAsync(ctx->mlp_m1.p, 0, kSelWeights * 4, ctx->stream));
    CUDA_TRY(cudaMemsetAsync(ctx->mlp_v2.p, 0, kSelWeights * 4, ctx->stream));
    const auto t0 = std::chrono::steady_clock::now();
    float loss_first = 0, loss_last = 0;
    for (int e = 0; e < o.epochs; ++e) {
        CUDA_TRY(cudaMemsetAsync(ctx->mlp_loss.p, 0, 4, ctx->stream));
        CUDA_TRY(mlp_loss_grad(ctx->mlp_w.as<float>(), ctx->mlp_x.as<float>(), ctx->mlp_y.as<float>(),
                               ctx->mlp_m.as<float>(), (uint32_t)n, (float)(1.0 / msum), ctx->mlp_grad.as<float>(),
                               ctx->mlp_loss.as<float>(), ctx->stream));
        if (e == 0 || e == o.epochs - 1) {
            float l = 0;
            CUDA_TRY(cudaMemcpyAsync(&l, ctx->mlp_loss.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
            CUDA_TRY(cudaStreamSynchronize(ctx->stream));
            (e == 0 ? loss_first : loss_last) = l;
            if (e == 0) loss_last = l;
        }
        CUDA_TRY(mlp_adam_step(ctx->mlp_w.as<float>(), ctx->mlp_grad.as<float>(), ctx->mlp_m1.as<float>(),
                               ctx->mlp_v2.as<float>(), o.learning_rate, o.weight_decay, (uint32_t)e + 1,
                               ctx->stream));
    }
    CUDA_TRY(cudaMemcpyAsync(sp.w, ctx->mlp_w.p, kSelWeights * 4, cudaMemcpyDeviceToHost, ctx->stream));
    CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < kSelWeights; ++i)
        if (!std::isfinite(sp.w[i])) {
            sp.has_weights = 0;
            return set_error(CFPQ_ERR_INVALID, "training diverged (lower the learning rate)");
        }
    sp.has_weights = 1;
    ctx->sel_dirty = true;
    if (report) {
        report->loss_first = loss_first;
        report->loss_last = loss_last;
        report->samples = (uint32_t)n;
        report->epochs = (uint32_t)o.epochs;
        report->ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return CFPQ_OK;
}

extern "C" int cfpq_autotune(cfpq_ctx *ctx, const cfpq_autotune_opts *opts, cfpq_selector_config *result,
                             float *timings) {
    TRY(use_ctx(ctx));
    static const uint32_t def_sizes[] = {2048, 8192};
    static const float def_dens[] = {0.002f, 0.02f, 0.1f, 0.3f, 0.6f};
    cfpq_autotune_opts o = {def_sizes, 2, def_dens, 5, 3, 1};
    if (opts) {
        o = *opts;
        if (!o.sizes || !o.nsizes || !o.densities || !o.ndensities)
            return set_error(CFPQ_ERR_INVALID, "empty size or density list");
        if (o.reps == 0) o.reps = 1;
    }
    for (size_t i = 0; i < o.nsizes; ++i)
        if (o.sizes[i] == 0 || o.sizes[i] > 32768)
            return set_error(CFPQ_ERR_INVALID, "autotune size %u out of range (1..32768)", o.sizes[i]);
    const int variants[3] = {CFPQ_VARIANT_LOP3, CFPQ_VARIANT_M4R, CFPQ_VARIANT_TC};
    std::vector<float> t(o.nsizes * o.ndensities * 3, -1.f);
    for (size_t si = 0; si < o.nsizes; ++si) {
        const uint32_t n = o.sizes[si];
        cfpq_matrix *a = nullptr, *b = nullptr, *c = nullptr;
        TRY(cfpq_matrix_create(ctx, n, &a));
        int rc = cfpq_matrix_create(ctx, n, &b);
        if (rc == CFPQ_OK) rc = cfpq_matrix_create(ctx, n, &c);
        for (size_t di = 0; di < o.ndensities && rc == CFPQ_OK; ++di) {
            cudaError_t e = launch_random_fill(a->d, o.densities[di], (uint64_t)o.seed * 1000003 + 2 * di, ctx->stream);
            if (e == cudaSuccess) e = launch_random_fill(b->d, o.densities[di], (uint64_t)o.seed * 1000003 + 2 * di + 1,
                                                         ctx->stream);
            if (e != cudaSuccess) {
                rc = set_error(CFPQ_ERR_CUDA, "random fill: %s", cudaGetErrorString(e));
                break;
            }
            for (int v = 0; v < 3 && rc == CFPQ_OK; ++v) {
                if (variants[v] == CFPQ_VARIANT_TC && !ctx->tc_grid) continue;
                float best = -1.f;
                for (uint32_t r = 0; r < o.reps && rc == CFPQ_OK; ++r) {
                    e = launch_clear_matrix(c->d, ctx->stream);
                    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev0, ctx->stream);
                    if (e != cudaSuccess) {
                        rc = set_error(CFPQ_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
                        break;
                    }
                    int changed = 0;
                    rc = cfpq_add_mul(ctx, c, a, b, variants[v], &changed);
                    if (rc != CFPQ_OK) break;
                    float ms = 0;
                    e = cudaEventRecord(ctx->ev1, ctx->stream);
                    if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev1);
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
                    if (e != cudaSuccess) {
                        rc = set_error(CFPQ_ERR_CUDA, "autotune timing: %s", cudaGetErrorString(e));
                        break;
                    }
                    best = best < 0 ? ms : std::min(best, ms);
                }
                t[(si * o.ndensities + di) * 3 + v] = best;
            }
        }
        if (a) cfpq_matrix_destroy(ctx, a);
        if (b) cfpq_matrix_destroy(ctx, b);
        if (c) cfpq_matrix_destroy(ctx, c);
        TRY(rc);
    }
    // Crossovers.  Random inputs populate every tile with mean population
    // density * 4096, so the density is the tile population the features see.
    SelectorParams &sp = ctx->sel;
    auto T = [&](size_t si, size_t di, int v) { return t[(si * o.ndensities + di) * 3 + v]; };
    // Four Russians: chosen when it beats LOP3 on every size at every density
    // whose tiles are dense (population above 96 bits)
    bool m4r_wins = true, any_dense = false;
    for (size_t si = 0; si < o.nsizes; ++si)
        for (size_t di = 0; di < o.ndensities; ++di)
            if (o.densities[di] * 4096.f > (float)kDenseTilePop) {
                any_dense = true;
                m4r_wins = m4r_wins && T(si, di, 1) > 0 && T(si, di, 1) < T(si, di, 0);
            }
    sp.m4r_min_dense = (any_dense && m4r_wins) ? 0.25f : 1.5f;
    // tensor cores: the smallest size at which TC beats both word-level
    // variants at every density whose tiles are dense sets tc_min_tiles (the
    // rule then takes TC where most P tiles are dense); no such size: never
    sp.tc_min_dense = 2.f;
    bool found = false;
    for (size_t si = 0; si < o.nsizes && ctx->tc_grid; ++si) {
        bool wins = false;
        for (size_t di = 0; di < o.ndensities; ++di) {
            if (o.densities[di] * 4096.f <= (float)kDenseTilePop) continue;
            const float tc = T(si, di, 2), w = std::min(T(si, di, 0), T(si, di, 1) > 0 ? T(si, di, 1) : 1e30f);
            wins = tc > 0 && tc < w;
            if (!wins) break;
        }
        if (wins && (!found || (o.sizes[si] + 63) / 64 < sp.tc_min_tiles)) {
            sp.tc_min_tiles = std::max<uint32_t>(1, (o.sizes[si] + 63) / 64);
            sp.tc_min_dense = 0.3f;
            found = true;
        }
    }
    sp.tc_min_occ = 0.2f;
    if (sp.mode == CFPQ_SELECT_FIXED) sp.mode = CFPQ_SELECT_HEURISTIC;
    ctx->sel_dirty = true;
    if (result) TRY(cfpq_selector_get_config(ctx, result));
    if (timings) memcpy(timings, t.data(), t.size() * sizeof(float));
    return CFPQ_OK;
}
