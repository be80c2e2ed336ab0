// B200 backend for the Matrix / MatricesEnv plug-in interface, used exactly
// like the reference's gpuMatrix / gpuMatricesEnv
// (cuda/naive-gpu/main.cpp:9-10, GpuMatrix.h:9-58):
//
//   grammar.intersection_with_graph<B200Matrix, B200MatricesEnv>(graph);
//
// Every matrix lives on the device (libcfpq_b200.so) from construction on.
// set_bit buffers coordinates on the host; environment_preprocessing scatters
// them on the device in one call per matrix.  environment_closure runs the
// whole fixpoint on the device (cfpq_closure), so the driver's host worklist
// is skipped; add_mul stays available for the worklist form.  After
// environment_postprocessing, get_bit reads a host mirror downloaded on first
// use and hash_count computes the result line on the device.
//
// Configuration (environment variables): CFPQ_DEVICE (default 0),
// CFPQ_DRIVER = engine | worklist (default engine), CFPQ_VARIANT = auto |
// plain | lop3 | m4r | tc (default auto), CFPQ_GRAPH = 0 (host loop) | 1
// (device: persistent kernel or CUDA graph) | 2 (CUDA graph), default 1;
// CFPQ_ORDER = 0 keeps vertex v at index v (default 1: a vertex order is
// suggested from the edges when the matrices are first uploaded).
//
// Errors throw std::runtime_error with the library's message (the reference
// prints and exits, cuda/naive-gpu/Multiplication.cu:10-17).
#ifndef CFPQ_B200_B200MATRIX_H
#define CFPQ_B200_B200MATRIX_H

#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "Matrix.h"
#include "cfpq_b200.h"

namespace cfpq_b200_detail {

inline void check(int rc, const char *what) {
    if (rc != CFPQ_OK) throw std::runtime_error(std::string(what) + ": " + cfpq_last_error());
}

inline int env_int(const char *name, int dflt) {
    const char *v = std::getenv(name);
    return v && *v ? std::atoi(v) : dflt;
}

// Process-wide context, created on first use (the reference keeps its device
// state in statics too, cuda/naive-gpu/GpuMatrix.h:15-16).
inline cfpq_ctx *context() {
    static cfpq_ctx *ctx = [] {
        cfpq_ctx *c = nullptr;
        check(cfpq_ctx_create(env_int("CFPQ_DEVICE", 0), &c), "cfpq_ctx_create");
        return c;
    }();
    return ctx;
}

inline int variant_from_env() {
    const char *v = std::getenv("CFPQ_VARIANT");
    if (!v || !*v || !std::strcmp(v, "auto")) return CFPQ_VARIANT_AUTO;
    if (!std::strcmp(v, "plain")) return CFPQ_VARIANT_PLAIN;
    if (!std::strcmp(v, "lop3")) return CFPQ_VARIANT_LOP3;
    if (!std::strcmp(v, "m4r")) return CFPQ_VARIANT_M4R;
    if (!std::strcmp(v, "tc")) return CFPQ_VARIANT_TC;
    if (!std::strcmp(v, "ntset")) return CFPQ_VARIANT_NTSET;
    throw std::runtime_error(std::string("unknown CFPQ_VARIANT ") + v);
}

inline int driver_from_env() {
    const char *v = std::getenv("CFPQ_DRIVER");
    if (!v || !*v || !std::strcmp(v, "engine")) return CFPQ_DRIVER_ENGINE;
    if (!std::strcmp(v, "worklist")) return CFPQ_DRIVER_WORKLIST;
    throw std::runtime_error(std::string("unknown CFPQ_DRIVER ") + v);
}

}  // namespace cfpq_b200_detail

class B200Matrix : public Matrix {
public:
    explicit B200Matrix(unsigned int n) : Matrix(n), n_(n) {
        cfpq_b200_detail::check(cfpq_matrix_create(cfpq_b200_detail::context(), n, &m_), "cfpq_matrix_create");
    }

    ~B200Matrix() override { cfpq_matrix_destroy(cfpq_b200_detail::context(), m_); }

    B200Matrix(const B200Matrix &) = delete;
    B200Matrix &operator=(const B200Matrix &) = delete;

    void set_bit(unsigned int row, unsigned col) override {
        if (row >= n_ || col >= n_) throw std::out_of_range("B200Matrix::set_bit: coordinate out of range");
        rows_.push_back(row);
        cols_.push_back(col);
        mirror_valid_ = false;
    }

    unsigned int get_bit(unsigned int row, unsigned col) override {
        if (row >= n_ || col >= n_) return 0;
        if (!mirror_valid_) download();
        const size_t wpr = (n_ + 63) / 64;
        return (unsigned int)((mirror_[(size_t)row * wpr + col / 64] >> (col % 64)) & 1u);
    }

    bool add_mul(Matrix *left, Matrix *right) override {
        auto *a = dynamic_cast<B200Matrix *>(left);
        auto *b = dynamic_cast<B200Matrix *>(right);
        if (!a || !b) throw std::invalid_argument("B200Matrix::add_mul: operands are not B200Matrix");
        a->flush();
        b->flush();
        flush();
        int changed = 0;
        cfpq_b200_detail::check(
            cfpq_add_mul(cfpq_b200_detail::context(), m_, a->m_, b->m_, cfpq_b200_detail::variant_from_env(), &changed),
            "cfpq_add_mul");
        mirror_valid_ = false;
        flushed_ = true;
        return changed != 0;
    }

    bool hash_count(unsigned long long *hash, unsigned long *count) override {
        flush();
        uint64_t h = 0, c = 0;
        cfpq_b200_detail::check(cfpq_matrix_hash_count(cfpq_b200_detail::context(), m_, &h, &c),
                                "cfpq_matrix_hash_count");
        *hash = h;
        *count = (unsigned long)c;
        return true;
    }

    // Scatter buffered set_bit coordinates on the device.
    void flush() {
        if (rows_.empty()) return;
        cfpq_b200_detail::check(
            cfpq_matrix_set_bits(cfpq_b200_detail::context(), m_, rows_.data(), cols_.data(), rows_.size()),
            "cfpq_matrix_set_bits");
        flushed_ = true;
        rows_.clear();
        cols_.clear();
        rows_.shrink_to_fit();
        cols_.shrink_to_fit();
    }

    void invalidate_mirror() { mirror_valid_ = false; }
    cfpq_matrix *handle() const { return m_; }
    unsigned int size() const { return n_; }

    // Coordinates set but not yet on the device, and whether the device
    // matrix is still empty (nothing flushed, no product written into it).
    const std::vector<uint32_t> &pending_rows() const { return rows_; }
    const std::vector<uint32_t> &pending_cols() const { return cols_; }
    bool device_empty() const { return !flushed_; }

    // Re-create the still empty device matrix in a vertex order (results are
    // still read in original vertex ids); the matrices of one order share it.
    void reorder(const std::shared_ptr<cfpq_order> &order) {
        if (flushed_) throw std::logic_error("B200Matrix::reorder: the matrix already holds bits on the device");
        cfpq_matrix *m = nullptr;
        cfpq_b200_detail::check(cfpq_matrix_create_ordered(cfpq_b200_detail::context(), n_, order.get(), &m),
                                "cfpq_matrix_create_ordered");
        cfpq_matrix_destroy(cfpq_b200_detail::context(), m_);
        m_ = m;
        order_ = order;
    }

private:
    void download() {
        flush();
        mirror_.assign((size_t)n_ * ((n_ + 63) / 64), 0);
        cfpq_b200_detail::check(cfpq_matrix_download_rows(cfpq_b200_detail::context(), m_, mirror_.data()),
                                "cfpq_matrix_download_rows");
        mirror_valid_ = true;
    }

    unsigned int n_;
    std::shared_ptr<cfpq_order> order_;  // released after the destructor body destroyed the matrix
    cfpq_matrix *m_ = nullptr;
    bool flushed_ = false;
    std::vector<uint32_t> rows_, cols_;
    std::vector<uint64_t> mirror_;
    bool mirror_valid_ = false;
};

class B200MatricesEnv : public MatricesEnv {
public:
    // Before the upload: when every matrix is still empty on the device, a
    // vertex order is suggested from all buffered coordinates (the matrix
    // index as the label: cfpq_order_suggest groups vertices by the labels on
    // their edges and orders each group breadth-first) and the matrices are
    // re-created in it, which gathers the occupied tiles (the same-generation
    // query at N = 8192: 55,222 -> 3,795 tiles of the result); then the
    // buffered coordinates are scattered.  CFPQ_ORDER=0 keeps vertex v at
    // index v.
    void environment_preprocessing(const std::vector<Matrix *> &matrices) override {
        if (cfpq_b200_detail::env_int("CFPQ_ORDER", 1) && !matrices.empty()) reorder_all(matrices);
        for (Matrix *m : matrices) as_b200(m)->flush();
    }

    bool environment_closure(const std::vector<cfpq_rule_entry> &rules, const std::vector<Matrix *> &matrices) override {
        std::vector<cfpq_rule> rs;
        rs.reserve(rules.size());
        for (const auto &r : rules) rs.push_back({r.first, r.second.first, r.second.second});
        std::vector<cfpq_matrix *> hs;
        hs.reserve(matrices.size());
        for (Matrix *m : matrices) hs.push_back(as_b200(m)->handle());
        cfpq_closure_opts o;
        std::memset(&o, 0, sizeof(o));
        o.driver = cfpq_b200_detail::driver_from_env();
        o.variant = cfpq_b200_detail::variant_from_env();
        o.use_graph = cfpq_b200_detail::env_int("CFPQ_GRAPH", 1);
        cfpq_b200_detail::check(cfpq_closure(cfpq_b200_detail::context(), rs.data(), rs.size(), hs.data(), hs.size(),
                                             &o, &stats_),
                                "cfpq_closure");
        for (Matrix *m : matrices) as_b200(m)->invalidate_mirror();
        return true;
    }

    void environment_postprocessing(const std::vector<Matrix *> &matrices) override {
        (void)matrices;
        cfpq_b200_detail::check(cfpq_ctx_synchronize(cfpq_b200_detail::context()), "cfpq_ctx_synchronize");
    }

    const cfpq_closure_stats &stats() const { return stats_; }

private:
    static void reorder_all(const std::vector<Matrix *> &matrices) {
        const unsigned int n = as_b200(matrices[0])->size();
        std::vector<uint32_t> src, lab, dst;
        for (size_t i = 0; i < matrices.size(); ++i) {
            B200Matrix *b = as_b200(matrices[i]);
            if (!b->device_empty() || b->size() != n) return;
            src.insert(src.end(), b->pending_rows().begin(), b->pending_rows().end());
            dst.insert(dst.end(), b->pending_cols().begin(), b->pending_cols().end());
            lab.insert(lab.end(), b->pending_rows().size(), (uint32_t)i);
        }
        if (src.empty() || n == 0) return;
        std::vector<uint32_t> perm(n);
        cfpq_b200_detail::check(cfpq_order_suggest(n, src.data(), lab.data(), dst.data(), src.size(), perm.data()),
                                "cfpq_order_suggest");
        bool identity = true;
        for (uint32_t v = 0; v < n && identity; ++v) identity = perm[v] == v;
        if (identity) return;
        cfpq_order *o = nullptr;
        cfpq_b200_detail::check(cfpq_order_create(cfpq_b200_detail::context(), n, perm.data(), &o), "cfpq_order_create");
        std::shared_ptr<cfpq_order> order(o, [](cfpq_order *p) { cfpq_order_destroy(cfpq_b200_detail::context(), p); });
        for (Matrix *m : matrices) as_b200(m)->reorder(order);
    }

    static B200Matrix *as_b200(Matrix *m) {
        auto *b = dynamic_cast<B200Matrix *>(m);
        if (!b) throw std::invalid_argument("B200MatricesEnv: matrix is not a B200Matrix");
        return b;
    }
    cfpq_closure_stats stats_{};
};

#endif  // CFPQ_B200_B200MATRIX_H
