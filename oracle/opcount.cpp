/*
 * CPU ORACLE, OPERATION-COUNTING BUILD — TEST / MEASUREMENT INFRASTRUCTURE ONLY.
 *
 * Compiles the oracle (hp_oracle.cpp, the restatement of the reference's element
 * residual) once more with every `double` replaced by a scalar type that counts its
 * arithmetic: one add, subtract, multiply or divide = 1 flop; sqrt and pow are
 * counted apart. oc_element_flops runs the element loop of tri_hp::rsdl(stage)
 * (tri_hp/nstage.cpp:52-73: ugtouht, element_rsdl, lftog of both parts) over every
 * element of a context and returns the counts per element, the algorithmic flops of
 * the reference's sum-factorised element residual. Used to write
 * profiles/flops_per_element.json (oracle/write_flop_table.py); never linked into the
 * shipped library.
 */
// every system header the oracle includes, before `double` is redefined (their include
// guards keep the oracle's own #includes from expanding them again)
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <vector>

namespace opc {
typedef double real_t;
struct Counts {
    unsigned long long flops, sqrts, pows;
};
static Counts g_cnt = {0, 0, 0};
struct Num {
    real_t v;
    Num() : v(0) {}
    Num(real_t x) : v(x) {}
    explicit operator real_t() const { return v; }
    Num &operator+=(Num o) { ++g_cnt.flops; v += o.v; return *this; }
    Num &operator-=(Num o) { ++g_cnt.flops; v -= o.v; return *this; }
    Num &operator*=(Num o) { ++g_cnt.flops; v *= o.v; return *this; }
    Num &operator/=(Num o) { ++g_cnt.flops; v /= o.v; return *this; }
};
inline Num operator+(Num a, Num b) { ++g_cnt.flops; return Num(a.v + b.v); }
inline Num operator-(Num a, Num b) { ++g_cnt.flops; return Num(a.v - b.v); }
inline Num operator*(Num a, Num b) { ++g_cnt.flops; return Num(a.v * b.v); }
inline Num operator/(Num a, Num b) { ++g_cnt.flops; return Num(a.v / b.v); }
inline Num operator-(Num a) { return Num(-a.v); }
inline Num operator+(Num a) { return a; }
inline bool operator<(Num a, Num b) { return a.v < b.v; }
inline bool operator>(Num a, Num b) { return a.v > b.v; }
inline bool operator<=(Num a, Num b) { return a.v <= b.v; }
inline bool operator>=(Num a, Num b) { return a.v >= b.v; }
inline bool operator==(Num a, Num b) { return a.v == b.v; }
inline bool operator!=(Num a, Num b) { return a.v != b.v; }
inline Num sqrt(Num a) { ++g_cnt.sqrts; return Num(std::sqrt(a.v)); }
inline Num fabs(Num a) { return Num(std::fabs(a.v)); }
inline Num pow(Num a, Num b) { ++g_cnt.pows; return Num(std::pow(a.v, b.v)); }
inline bool isnan(Num a) { return std::isnan(a.v); }
}  // namespace opc

namespace std {
inline opc::Num sqrt(opc::Num a) { return opc::sqrt(a); }
inline opc::Num fabs(opc::Num a) { return opc::fabs(a); }
inline opc::Num pow(opc::Num a, opc::Num b) { return opc::pow(a, b); }
inline opc::Num pow(opc::Num a, int b) { return opc::pow(a, opc::Num((double)b)); }
inline bool isnan(opc::Num a) { return opc::isnan(a); }
// a double literal beside a counted value (std::max(gam, 0.1))
inline opc::Num max(opc::Num a, opc::real_t b) { return a.v < b ? opc::Num(b) : a; }
inline opc::Num min(opc::Num a, opc::real_t b) { return b < a.v ? opc::Num(b) : a; }
}  // namespace std

#define double opc::Num
#include "hp_oracle.cpp"
#undef double

extern "C" {
// Flops per element of the element loop of rsdl(stage) over every element of c; out[0]
// = add/sub/mul/div count, out[1] = sqrt count, out[2] = pow count, each per element.
void oc_element_flops(or_ctx *c, int stage, opc::real_t *out) {
    opc::Num lf_re[3][HP_MXTM], lf_im[3][HP_MXTM];
    std::vector<opc::Num> rv(c->resv.size()), rs(c->ress.size()), ri(c->resi.size());
    opc::g_cnt = {0, 0, 0};
    for (int tind = 0; tind < c->ntri; ++tind) {
        ugtouht(c, tind);
        if (c->ph.physics == HP_PHYS_INS) element_rsdl_ins(c, tind, stage, lf_re, lf_im);
        else element_rsdl_cd(c, tind, stage, lf_re, lf_im);
        lftog(c, tind, lf_im, rv.data(), rs.data(), ri.data());
        lftog(c, tind, lf_re, rv.data(), rs.data(), ri.data());
    }
    out[0] = (opc::real_t)opc::g_cnt.flops / c->ntri;
    out[1] = (opc::real_t)opc::g_cnt.sqrts / c->ntri;
    out[2] = (opc::real_t)opc::g_cnt.pows / c->ntri;
}
}
