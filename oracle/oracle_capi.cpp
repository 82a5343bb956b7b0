// oracle_capi.cpp -- TEST INFRASTRUCTURE ONLY: C entry points of the CPU
// oracle (tslb_oracle.hpp) for the parity tests and the CPU baseline.
// Arrays cross the boundary as FP64, interior nodes only, Fortran order
// (x fastest); the oracle computes in float (fp64 == 0) or double.
#include <memory>
#include <string>

#include "tslb_oracle.hpp"

namespace {

struct Handle {
    bool fp64;
    std::unique_ptr<orc::Oracle<float>> o32;
    std::unique_ptr<orc::Oracle<double>> o64;
};

template <class R, class Fn>
int with(Handle* h, Fn fn) {
    if (!h) return TSLB_ERR_ARG;
    if constexpr (std::is_same<R, float>::value) return fn(*h->o32);
    else return fn(*h->o64);
}

template <class R>
int set_moments_t(orc::Oracle<R>& o, const double* in) {
    size_t n = size_t(o.nx) * o.ny * o.nz;
    std::vector<R> m[orc::NFIELD];
    for (int c = 0; c < orc::NFIELD; ++c) {
        m[c].resize(n);
        for (size_t s = 0; s < n; ++s) m[c][s] = R(in[size_t(c) * n + s]);
    }
    o.set_moments(m);
    return TSLB_OK;
}

template <class R>
int get_moments_t(orc::Oracle<R>& o, double* out) {
    std::vector<R> m[orc::NFIELD];
    o.get_moments(m);
    size_t n = size_t(o.nx) * o.ny * o.nz;
    for (int c = 0; c < orc::NFIELD; ++c)
        for (size_t s = 0; s < n; ++s) out[size_t(c) * n + s] = double(m[c][s]);
    return TSLB_OK;
}

template <class R>
int set_pops_t(orc::Oracle<R>& o, const double* f, const double* g) {
    size_t n = size_t(o.nx) * o.ny * o.nz;
    std::vector<R> fv(27 * n), gv(size_t(o.nq_g) * n);
    for (size_t s = 0; s < fv.size(); ++s) fv[s] = R(f[s]);
    for (size_t s = 0; s < gv.size(); ++s) gv[s] = R(g[s]);
    o.set_pops(fv, gv);
    return TSLB_OK;
}

template <class R>
int get_normals_t(orc::Oracle<R>& o, double* out) {
    std::vector<R> nn[3];
    o.get_normals(nn);
    size_t n = size_t(o.nx) * o.ny * o.nz;
    for (int c = 0; c < 3; ++c)
        for (size_t s = 0; s < n; ++s) out[size_t(c) * n + s] = double(nn[c][s]);
    return TSLB_OK;
}

template <class R>
int set_inlet_t(orc::Oracle<R>& o, int face, const double* in) {
    auto& pl = o.inlet[face];
    for (size_t s = 0; s < pl.size(); ++s) pl[s] = R(in[s]);
    return TSLB_OK;
}

template <class R>
int set_dtau_t(orc::Oracle<R>& o, const double* in) {
    size_t n = size_t(o.nx) * o.ny * o.nz;
    if (!in) { o.dtau.clear(); return TSLB_OK; }
    o.dtau.resize(n);
    for (size_t s = 0; s < n; ++s) o.dtau[s] = R(in[s]);
    return TSLB_OK;
}

}  // namespace

extern "C" {

void* orc_create(const tslb_params* p, int nx, int ny, int nz, int fp64) {
    if (!p || nx < 1 || ny < 1 || nz < 1) return nullptr;
    auto* h = new Handle();
    h->fp64 = fp64 != 0;
    if (h->fp64) h->o64.reset(new orc::Oracle<double>(*p, nx, ny, nz));
    else h->o32.reset(new orc::Oracle<float>(*p, nx, ny, nz));
    return h;
}

void orc_destroy(void* hp) { delete static_cast<Handle*>(hp); }

#define ORC_DISPATCH(hp, CALL)                                                   \
    Handle* h = static_cast<Handle*>(hp);                                        \
    if (!h) return TSLB_ERR_ARG;                                                 \
    if (h->fp64) { auto& o = *h->o64; return CALL; }                             \
    else { auto& o = *h->o32; return CALL; }

int orc_set_moments(void* hp, const double* in) { ORC_DISPATCH(hp, set_moments_t(o, in)); }
int orc_get_moments(void* hp, double* out) { ORC_DISPATCH(hp, get_moments_t(o, out)); }
int orc_set_pops(void* hp, const double* f, const double* g) { ORC_DISPATCH(hp, set_pops_t(o, f, g)); }
int orc_get_normals(void* hp, double* out) { ORC_DISPATCH(hp, get_normals_t(o, out)); }
int orc_set_inlet(void* hp, int face, const double* in) {
    if (face < 0 || face > 5) return TSLB_ERR_ARG;
    ORC_DISPATCH(hp, set_inlet_t(o, face, in));
}
int orc_set_dtau(void* hp, const double* in) { ORC_DISPATCH(hp, set_dtau_t(o, in)); }
int orc_set_isfluid(void* hp, const unsigned char* in) {
    ORC_DISPATCH(hp, (([&]() {
        if (!in) { o.isfluid.clear(); return int(TSLB_OK); }
        o.isfluid.assign(in, in + size_t(o.nx) * o.ny * o.nz);
        return int(TSLB_OK);
    })()));
}
int orc_step(void* hp, int nsteps) {
    ORC_DISPATCH(hp, (([&]() { for (int s = 0; s < nsteps; ++s) o.step(); return int(TSLB_OK); })()));
}
int orc_reduce(void* hp, double* out) {
    ORC_DISPATCH(hp, (([&]() { o.reduce(out); return int(TSLB_OK); })()));
}

}  // extern "C"
