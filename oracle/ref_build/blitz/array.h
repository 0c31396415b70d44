/*
 * Minimal container subset with the blitz++ names that the reference's
 * tri_basis and tet_basis sources use outside their BZ_DEBUG blocks: TinyVector,
 * TinyMatrix (fixed size, row-major), Array<T,R> (R = 1..4, row-major,
 * resizable, fill by scalar assignment) and Range::all() for the one column
 * assignment tet_basis makes. Every allocation carries PAD spare elements: the
 * reference's tet_basis::lumpinv writes idiag(0) for p < 4 where idiag has no
 * element (blitz without bounds checks lets that pass), and the spare elements
 * absorb such writes.
 *
 * TEST INFRASTRUCTURE ONLY. This header exists so that the reference's own
 * tri_basis/*.cpp and tet_basis/*.cpp files compile unmodified, where they lie,
 * into the checker libraries under oracle/_ref/. Nothing in the shipped library
 * includes it.
 */
#ifndef HPB_ORACLE_BLITZ_SHIM_H
#define HPB_ORACLE_BLITZ_SHIM_H

#include <vector>
#include <cstddef>
#include <iostream>

namespace blitz {

/* blitz++ makes the std names visible through "using namespace blitz". */
using namespace std;

template <class T, int N>
class TinyVector {
    T d_[N];

public:
    TinyVector() {}
    T &operator()(int i) { return d_[i]; }
    const T &operator()(int i) const { return d_[i]; }
    T *data() { return d_; }
    const T *data() const { return d_; }
    TinyVector &operator=(T v) {
        for (int i = 0; i < N; ++i) d_[i] = v;
        return *this;
    }
};

template <class T, int N, int M>
class TinyMatrix {
    T d_[N * M];

public:
    TinyMatrix() {}
    T &operator()(int i, int j) { return d_[i * M + j]; }
    const T &operator()(int i, int j) const { return d_[i * M + j]; }
    T *data() { return d_; }
    const T *data() const { return d_; }
    TinyMatrix &operator=(T v) {
        for (int i = 0; i < N * M; ++i) d_[i] = v;
        return *this;
    }
};

struct Range {
    static Range all() { return Range(); }
};

template <class T, int R>
class Array {
    static constexpr size_t PAD = 16;
    std::vector<T> v_;
    int e_[4] = {0, 0, 0, 0};

public:
    /* column view of a rank-2 array: a(Range::all(), j) = value */
    struct Column {
        Array *a;
        int j;
        Column &operator=(T v) {
            for (int i = 0; i < a->e_[0]; ++i) (*a)(i, j) = v;
            return *this;
        }
    };
    Column operator()(Range, int j) { return Column{this, j}; }
    Array &operator=(T v) {
        for (size_t i = 0; i + PAD < v_.size(); ++i) v_[i] = v;
        return *this;
    }
    Array() {}
    explicit Array(int n0) { resize(n0); }
    Array(int n0, int n1) { resize(n0, n1); }
    Array(int n0, int n1, int n2) { resize(n0, n1, n2); }
    Array(int n0, int n1, int n2, int n3) { resize(n0, n1, n2, n3); }
    void resize(int n0) {
        e_[0] = n0; e_[1] = 1; e_[2] = 1; e_[3] = 1;
        v_.assign((size_t)n0 + PAD, T());
    }
    void resize(int n0, int n1) {
        e_[0] = n0; e_[1] = n1; e_[2] = 1; e_[3] = 1;
        v_.assign((size_t)n0 * n1 + PAD, T());
    }
    void resize(int n0, int n1, int n2) {
        e_[0] = n0; e_[1] = n1; e_[2] = n2; e_[3] = 1;
        v_.assign((size_t)n0 * n1 * n2 + PAD, T());
    }
    void resize(int n0, int n1, int n2, int n3) {
        e_[0] = n0; e_[1] = n1; e_[2] = n2; e_[3] = n3;
        v_.assign((size_t)n0 * n1 * n2 * n3 + PAD, T());
    }
    int extent(int d) const { return e_[d]; }
    T &operator()(int i) { return v_[i]; }
    const T &operator()(int i) const { return v_[i]; }
    T &operator()(int i, int j) { return v_[(size_t)i * e_[1] + j]; }
    const T &operator()(int i, int j) const { return v_[(size_t)i * e_[1] + j]; }
    T &operator()(int i, int j, int k) { return v_[((size_t)i * e_[1] + j) * e_[2] + k]; }
    const T &operator()(int i, int j, int k) const { return v_[((size_t)i * e_[1] + j) * e_[2] + k]; }
    T &operator()(int i, int j, int k, int l) { return v_[(((size_t)i * e_[1] + j) * e_[2] + k) * e_[3] + l]; }
    const T &operator()(int i, int j, int k, int l) const {
        return v_[(((size_t)i * e_[1] + j) * e_[2] + k) * e_[3] + l];
    }
    T *data() { return v_.data(); }
    const T *data() const { return v_.data(); }
};

}  // namespace blitz

#endif
