// Matrix / MatricesEnv plug-in interface, source-compatible with the
// reference's cfpq-cpp/Matrix.h:7-37: a backend derives from Matrix and
// (optionally) MatricesEnv and is selected with
// Grammar::intersection_with_graph<MyMatrix, MyEnv>(graph).
//
// Two optional hooks are added; both have defaults that keep existing
// backends working unchanged:
//   MatricesEnv::environment_closure -- called by the driver after
//     environment_preprocessing; a backend that runs the whole fixpoint itself
//     returns true and the driver skips its host worklist.
//   Matrix::hash_count -- lets print_results take the result line from the
//     backend instead of n^2 get_bit calls; default returns false.
#ifndef CFPQ_B200_MATRIX_H
#define CFPQ_B200_MATRIX_H

#include <utility>
#include <vector>

class Matrix {
public:
    explicit Matrix(unsigned int n) { (void)n; }

    virtual ~Matrix() = default;

    virtual void set_bit(unsigned int row, unsigned col) = 0;

    virtual unsigned int get_bit(unsigned int row, unsigned col) = 0;

    // this |= left * right over (OR, AND); true if any bit of this changed.
    virtual bool add_mul(Matrix *left, Matrix *right) = 0;

    // Optional: the result line's hash and count (Grammar.cpp:84-97 semantics).
    virtual bool hash_count(unsigned long long *hash, unsigned long *count) {
        (void)hash;
        (void)count;
        return false;
    }

    static unsigned int toBoolVector(unsigned int number) { return 1u << number; }

    static unsigned char toBoolVector8(unsigned int number) { return (unsigned char)(1u << number); }
};

// (head, (body1, body2)) -- the driver's rule representation.
using cfpq_rule_entry = std::pair<unsigned int, std::pair<unsigned int, unsigned int>>;

class MatricesEnv {
public:
    MatricesEnv() = default;

    virtual ~MatricesEnv() = default;

    virtual void environment_preprocessing(const std::vector<Matrix *> &matrices) { (void)matrices; }

    // Optional: run the whole closure.  Return true if done (the driver then
    // skips its worklist), false to let the driver run add_mul one at a time.
    virtual bool environment_closure(const std::vector<cfpq_rule_entry> &rules,
                                     const std::vector<Matrix *> &matrices) {
        (void)rules;
        (void)matrices;
        return false;
    }

    virtual void environment_postprocessing(const std::vector<Matrix *> &matrices) { (void)matrices; }
};

#endif  // CFPQ_B200_MATRIX_H
