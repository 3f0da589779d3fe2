// Host-side preparation / post-processing of the propagator (see host_ops.h).
//
// These routines keep the reference's floating-point semantics where they
// are observable in the results: the reference stores `data_t` (float) but
// calls the global double overloads of sqrt/cos/pow/round/ceil on float
// arguments, so several expressions are evaluated in double and rounded to
// float once.  Each function states the reference lines it follows.
#include "host_ops.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace fwi {

namespace {
const float kH[4] = {(float)(17.0 / 48), (float)(59.0 / 48), (float)(43.0 / 48), (float)(49.0 / 48)};

inline float hcoef(int n, int i)
{
    // misc.cpp:4-9
    if (i < 4) return kH[i];
    if (i >= n - 4) return kH[n - 1 - i];
    return 1.f;
}

// Element-wise loops and min / max reductions over the model, in parallel
// (min and max are exact, so the results do not depend on the split).
inline float fmin_range(const float *p, int64_t n)
{
    float v = p[0];
#pragma omp parallel for reduction(min : v) schedule(static)
    for (int64_t i = 1; i < n; i++) v = std::min(v, p[i]);
    return v;
}
inline float fmax_range(const float *p, int64_t n)
{
    float v = p[0];
#pragma omp parallel for reduction(max : v) schedule(static)
    for (int64_t i = 1; i < n; i++) v = std::max(v, p[i]);
    return v;
}
inline void clip_range(float *p, int64_t n, float lo, float hi)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) p[i] = std::max(lo, std::min(hi, p[i]));
}
}  // namespace

TimeAxis analyze_model(std::vector<float> &model, int nmodels, int nx, int ny, int nz, float dx, float dy, float dz,
                       int nt_data, float dt_data, const fwi_param &p)
{
    const int64_t n = (int64_t)nx * ny * nz;
    float *m = model.data();
    TimeAxis ta{};
    if (nmodels >= 3) {
        if (nmodels == 6) {
            // Thomsen-delta admissibility clip; the reference scans the first nx*nz
            // samples only (we_op.cpp:274-286), reproduced as is.
            const float *pvp = m, *pvs = m + n;
            float *pdel = m + 3 * n;
            for (int64_t i = 0; i < (int64_t)nx * nz; i++) {
                const float val1 = (float)(-0.5 * (1 - pvs[i] * pvs[i] / (pvp[i] * pvp[i])));
                const float val2 = (float)(2.0 / (pvp[i] * pvp[i] / (pvs[i] * pvs[i]) - 1));
                if (pdel[i] < val1) pdel[i] = (float)(0.9999 * val1);
                else if (pdel[i] > val2) pdel[i] = (float)(0.9999 * val2);
            }
        }
        if (!p.soft_clip) {
            clip_range(m, n, p.vpmin, p.vpmax);
            clip_range(m + n, n, p.vsmin, p.vsmax);
            clip_range(m + 2 * n, n, p.rhomin, p.rhomax);
            if (nmodels == 6) {
                clip_range(m + 3 * n, n, p.deltamin, p.deltamax);
                clip_range(m + 4 * n, n, p.epsilonmin, p.epsilonmax);
                clip_range(m + 5 * n, n, p.gammamin, p.gammamax);
            }
            // vs <= vp/sqrt(2) (we_op.cpp:331-341)
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; i++)
                if ((double)m[i] < std::sqrt(2.0) * (double)m[n + i]) m[n + i] = (float)((double)m[i] / std::sqrt(2.0001));
        }
        ta.vmax = fmax_range(m, n);
        ta.vmin = fmin_range(m + n, n);
        if (nmodels == 6) {
            float t = (float)((double)m[0] * std::sqrt((double)(1 + 2 * m[4 * n])));
#pragma omp parallel for reduction(max : t) schedule(static)
            for (int64_t i = 1; i < n; i++) {
                const float v = (float)((double)m[i] * std::sqrt((double)(1 + 2 * m[4 * n + i])));
                t = std::max(t, v);
            }
            ta.vmax = std::max(t, ta.vmax);
        }
    } else {
        clip_range(m, n, p.vpmin, p.vpmax);
        clip_range(m + n, n, p.rhomin, p.rhomax);
        ta.vmax = fmax_range(m, n);
        ta.vmin = fmin_range(m, n);
    }

    // time step (we_op.cpp:417-432)
    const float dmin = std::min(std::min(dx, dy), dz);
    float dt = p.dt, courant = p.courant;
    if (dt == 0) {
        dt = courant * dmin / ta.vmax;
    } else if (dt > 0) {
        dt = std::min(dt, dt_data);
        courant = dt * ta.vmax / dmin;
    } else {
        dt = courant * dmin / ta.vmax;
        if (dt_data > dt) dt = (float)((double)dt_data / std::ceil((double)(dt_data / dt)));
        else dt = dt_data;
        courant = dt * ta.vmax / dmin;
    }
    const float tmax = (nt_data - 1) * dt_data;
    ta.nt = (int)(std::round((double)(tmax / dt)) + 1);
    ta.dt = dt;
    ta.courant = courant;
    ta.sub = p.sub < 0 ? (int)std::round((double)(dt_data / dt)) : p.sub;
    return ta;
}

void convert_model(std::vector<float> &model, int nmodels, int64_t n)
{
    float *m = model.data();
    float *p0 = m, *p1 = m + n, *p2 = m + 2 * n;
    if (nmodels == 2) {
        // we_op.cpp:1539-1545
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) {
            p0[i] = p1[i] * p0[i] * p0[i];
            p1[i] = (float)(1.0 / p1[i]);
        }
        return;
    }
    float *p3 = m + 3 * n, *p5 = m + 5 * n;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        p0[i] = p2[i] * (p0[i] * p0[i] - 2 * p1[i] * p1[i]);  // lambda
        p1[i] = p2[i] * p1[i] * p1[i];                          // mu
        if (nmodels == 6) {
            // c13 and c66 (we_op.cpp:1093-1094)
            p3[i] = (float)(std::sqrt((double)(2 * (p0[i] + 2 * p1[i]) * (p0[i] + p1[i]) * p3[i] +
                                               (p0[i] + p1[i]) * (p0[i] + p1[i]))) -
                            p1[i]);
            p5[i] = (1 + 2 * p5[i]) * p1[i];
        }
    }
}

std::vector<float> expand_wavelet(const float *w, int ncomp_in, int nt, int nmodels, const fwi_param &p)
{
    int nscomp = nmodels == 2 ? 1 : (p.mt ? 6 : 3);
    if (ncomp_in != 1) {
        if (ncomp_in != nscomp) throw std::invalid_argument("wavelet has the wrong number of components");
        return std::vector<float>(w, w + (size_t)ncomp_in * nt);
    }
    std::vector<float> out((size_t)nscomp * nt);
    if (nscomp == 1) {
        std::memcpy(out.data(), w, sizeof(float) * nt);
    } else if (nscomp == 3) {
        // vector force (we_op.cpp:169-175)
        for (int it = 0; it < nt; it++) {
            out[it] = (float)(w[it] * std::cos((double)p.fangle) * std::cos((double)p.fazimuth));
            out[nt + it] = (float)(w[it] * std::cos((double)p.fangle) * std::sin((double)p.fazimuth));
            out[2 * nt + it] = (float)(w[it] * std::sin((double)p.fangle));
        }
    } else {
        const float mm[6] = {p.mxx, p.myy, p.mzz, p.mxy, p.mxz, p.myz};
        for (int c = 0; c < 6; c++)
            for (int it = 0; it < nt; it++) out[(size_t)c * nt + it] = w[it] * mm[c];
    }
    return out;
}

namespace {
inline float sincf_ref(float x)
{
    // operator.cpp:418-421 (argument rounded to float, sin in double)
    if (x == 0.0) return 1.0f;
    return (float)(std::sin((double)x) / x);
}
}  // namespace

namespace {
// Sinc-resampler taps of one output sample: the weights depend on the two time
// axes only, so they are evaluated once (with the reference's mixed float /
// double semantics, operator.cpp:472-520) and applied to every trace.
struct SincTaps {
    std::vector<int> first, count;  // per output sample
    std::vector<float> s;           // windowed-sinc factor (float, as returned by sinc())
    std::vector<double> win;        // cosine window (double)
};
SincTaps sinc_taps(int hl, int nt_in, float dt_in, int nt_out, float dt_out)
{
    SincTaps T;
    T.first.resize(nt_out);
    T.count.resize(nt_out);
    const float a = 0.5f;
    for (int itd = 0; itd < nt_out; itd++) {
        const float t = itd * dt_out;
        const int itm0 = (int)std::floor((double)(t / dt_in));
        const int lo = std::max(0, itm0 - hl + 1), hi = std::min(nt_in - 1, itm0 + hl);
        T.first[itd] = lo;
        T.count[itd] = std::max(0, hi - lo + 1);
        for (int itm = lo; itm <= hi; itm++) {
            T.s.push_back(sincf_ref((float)(M_PI * (t - itm * dt_in) / dt_in)));
            T.win.push_back(a + (1 - a) * std::cos(M_PI * (itm - t / dt_in) / hl));
        }
    }
    return T;
}
}  // namespace

void sinc_resample_taps(int hl, int nt_in, float dt_in, int nt_out, float dt_out, std::vector<int> &first,
                        std::vector<int> &count, std::vector<float> &s, std::vector<double> &win)
{
    SincTaps T = sinc_taps(hl, nt_in, dt_in, nt_out, dt_out);
    first = std::move(T.first);
    count = std::move(T.count);
    s = std::move(T.s);
    win = std::move(T.win);
}

void resample_forward(bool sinc, int hl, const float *in, int nt_in, float dt_in, float *out, int nt_out, float dt_out,
                      int ntr)
{
    if (!sinc) {
        // operator.cpp:424-444
#pragma omp parallel for schedule(static)
        for (int ix = 0; ix < ntr; ix++)
            for (int it = 0; it < nt_out; it++) {
                const int i = std::min(nt_in - 1, (int)std::floor((double)(it * dt_out / dt_in)));
                const int j = std::min(nt_in - 1, (int)std::ceil((double)(it * dt_out / dt_in)));
                const float wj = (it * dt_out - i * dt_in) / dt_in;
                const float wi = 1 - wj;
                out[(size_t)ix * nt_out + it] = wi * in[(size_t)ix * nt_in + i] + wj * in[(size_t)ix * nt_in + j];
            }
        return;
    }
    const SincTaps T = sinc_taps(hl, nt_in, dt_in, nt_out, dt_out);
    std::vector<size_t> off(nt_out + 1, 0);
    for (int itd = 0; itd < nt_out; itd++) off[itd + 1] = off[itd] + T.count[itd];
#pragma omp parallel for schedule(static)
    for (int ix = 0; ix < ntr; ix++) {
        const float *src = in + (size_t)ix * nt_in;
        for (int itd = 0; itd < nt_out; itd++) {
            float acc = 0.f;
            for (int k = 0; k < T.count[itd]; k++) {
                const size_t q = off[itd] + k;
                acc = (float)((double)acc + (double)(src[T.first[itd] + k] * T.s[q]) * T.win[q]);
            }
            out[(size_t)ix * nt_out + itd] = acc;
        }
    }
}

void resample_adjoint(bool sinc, int hl, float *in, int nt_in, float dt_in, const float *out, int nt_out, float dt_out,
                      int ntr)
{
    // accumulates into `in` (callers zero it first for add=false), operator.cpp:446-520
    if (!sinc) {
#pragma omp parallel for schedule(static)
        for (int ix = 0; ix < ntr; ix++)
            for (int it = 0; it < nt_out; it++) {
                const int i = std::min(nt_in - 1, (int)std::floor((double)(it * dt_out / dt_in)));
                const int j = std::min(nt_in - 1, (int)std::ceil((double)(it * dt_out / dt_in)));
                const float wj = (it * dt_out - i * dt_in) / dt_in;
                const float wi = 1 - wj;
                in[(size_t)ix * nt_in + i] += wi * out[(size_t)ix * nt_out + it];
                in[(size_t)ix * nt_in + j] += wj * out[(size_t)ix * nt_out + it];
            }
        return;
    }
    const SincTaps T = sinc_taps(hl, nt_in, dt_in, nt_out, dt_out);
    std::vector<size_t> off(nt_out + 1, 0);
    for (int itd = 0; itd < nt_out; itd++) off[itd + 1] = off[itd] + T.count[itd];
#pragma omp parallel for schedule(static)
    for (int ix = 0; ix < ntr; ix++) {
        float *dst = in + (size_t)ix * nt_in;
        const float *src = out + (size_t)ix * nt_out;
        for (int itd = 0; itd < nt_out; itd++)
            for (int k = 0; k < T.count[itd]; k++) {
                const size_t q = off[itd] + k;
                float &d = dst[T.first[itd] + k];
                d = (float)((double)d + (double)(src[itd] * T.s[q]) * T.win[q]);
            }
    }
}

void apply_ht(bool inv, const float *in, float *out, int ntr, int nt, float dt)
{
    // misc.cpp:44-68 (in-place safe)
    for (int ix = 0; ix < ntr; ix++) {
        const size_t i1 = (size_t)ix * nt;
        if (!inv) {
            out[i1] = (float)(in[i1] * 0.5 * dt);
            for (int it = 1; it < nt - 1; it++) out[i1 + it] = in[i1 + it] * dt;
            out[i1 + nt - 1] = (float)(in[i1 + nt - 1] * 0.5 * dt);
        } else {
            out[i1] = (float)(in[i1] / (0.5 * dt));
            for (int it = 1; it < nt - 1; it++) out[i1 + it] = in[i1 + it] / dt;
            out[i1 + nt - 1] = (float)(in[i1 + nt - 1] / (0.5 * dt));
        }
    }
}

void apply_dt(bool adj, const float *in, float *out, int ntr, int nt, float dt)
{
    // misc.cpp:70-94 (out must not alias in)
    for (int ix = 0; ix < ntr; ix++) {
        const size_t i1 = (size_t)ix * nt;
        if (!adj) {
            out[i1] = (in[i1 + 1] - in[i1]) / dt;
            for (int it = 1; it < nt - 1; it++) out[i1 + it] = (in[i1 + it + 1] - in[i1 + it - 1]) / (2 * dt);
            out[i1 + nt - 1] = (in[i1 + nt - 1] - in[i1 + nt - 2]) / dt;
        } else {
            out[i1] = (in[i1 + 1] + in[i1]) / dt;
            for (int it = 1; it < nt - 1; it++) out[i1 + it] = (in[i1 + it + 1] - in[i1 + it - 1]) / (2 * dt);
            out[i1 + nt - 1] = (-in[i1 + nt - 1] - in[i1 + nt - 2]) / dt;
        }
    }
}

PointOp make_delta(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                   const std::vector<Loc> &loc, bool derivative)
{
    // delta_m3 / ddelta_m3 ::findIndicesWeights (injector.cpp:3-84, 142-238)
    PointOp op;
    op.npts = (int)loc.size();
    op.derivative = derivative;
    const int nw = op.nw();
    op.xind.assign(3 * op.npts, 0);
    op.yind.assign(3 * op.npts, 0);
    op.zind.assign(3 * op.npts, 0);
    op.xw.assign((size_t)2 * nw * op.npts, 0.f);
    op.yw.assign((size_t)2 * nw * op.npts, 0.f);
    op.zw.assign((size_t)2 * nw * op.npts, 0.f);
    auto axis = [&](float l, float o, float d, int n, int *ind, float *w) {
        int piv = (int)std::round((l - o) / d);
        if (piv == 0) piv = 1;
        if (piv == n - 1) piv = n - 2;
        ind[0] = piv - 1;
        ind[1] = piv;
        ind[2] = piv + 1;
        const float a = (l - d * piv - o) / d;
        const double a2 = std::pow((double)a, 2);
        float *wi = w, *we = w + nw;  // injection, extraction
        wi[0] = (float)((a2 - a) / (2 * d * hcoef(n, ind[0])));
        wi[1] = (float)((-a2 + 1) / (d * hcoef(n, ind[1])));
        wi[2] = (float)((a2 + a) / (2 * d * hcoef(n, ind[2])));
        we[0] = (float)((a2 - a) / 2);
        we[1] = (float)(-a2 + 1);
        we[2] = (float)((a2 + a) / 2);
        if (nw == 6) {
            wi[3] = (1 - 2 * a) / (2 * d * d * hcoef(n, ind[0]));
            wi[4] = 2 * a / (d * d * hcoef(n, ind[1]));
            wi[5] = (-1 - 2 * a) / (2 * d * d * hcoef(n, ind[2]));
            we[3] = (1 - 2 * a) / (2 * d);
            we[4] = 2 * a / (d);
            we[5] = (-1 - 2 * a) / (2 * d);
        }
    };
    for (int r = 0; r < op.npts; r++) {
        axis(loc[r].x, ox, dx, nx, &op.xind[3 * r], &op.xw[(size_t)2 * nw * r]);
        axis(loc[r].y, oy, dy, ny, &op.yind[3 * r], &op.yw[(size_t)2 * nw * r]);
        axis(loc[r].z, oz, dz, nz, &op.zind[3 * r], &op.zw[(size_t)2 * nw * r]);
    }
    return op;
}

InjTable injection_table(const PointOp &op, int nx, int ny, int nz, int ncomp_field)
{
    // delta_m3::inject (injector.cpp:86-116): u_c += (yw*xw*zw) * src[c][r][it]
    // ddelta_m3::inject (injector.cpp:240-278): moment-tensor derivative weights,
    // components (xx,yy,zz,xy,xz,yz) = traces 0..5 of each point.
    InjTable t;
    const int nw = op.nw();
    for (int r = 0; r < op.npts; r++) {
        const float *xw = &op.xw[(size_t)2 * nw * r], *yw = &op.yw[(size_t)2 * nw * r], *zw = &op.zw[(size_t)2 * nw * r];
        for (int iy = 0; iy < 3; iy++)
            for (int ix = 0; ix < 3; ix++)
                for (int iz = 0; iz < 3; iz++) {
                    const int64_t g =
                        ((int64_t)op.yind[3 * r + iy] * nx + op.xind[3 * r + ix]) * nz + op.zind[3 * r + iz];
                    if (!op.derivative) {
                        const float w = yw[iy] * xw[ix] * zw[iz];
                        for (int c = 0; c < ncomp_field; c++) {
                            t.gidx[c].push_back(g);
                            t.trace[c].push_back(c * op.npts + r);
                            t.w[c].push_back(w);
                        }
                    } else {
                        static const int ic[3][3] = {{0, 3, 4}, {3, 1, 5}, {4, 5, 2}};
                        const float wx = -xw[ix + 3] * yw[iy] * zw[iz];
                        const float wy = -xw[ix] * yw[iy + 3] * zw[iz];
                        const float wz = -xw[ix] * yw[iy] * zw[iz + 3];
                        for (int c = 0; c < 3; c++) {
                            const float ws[3] = {wx, wy, wz};
                            for (int k = 0; k < 3; k++) {
                                t.gidx[c].push_back(g);
                                t.trace[c].push_back(ic[c][k] * op.npts + r);
                                t.w[c].push_back(ws[k]);
                            }
                        }
                    }
                }
    }
    return t;
}

ExtTable extraction_table(const PointOp &op, int nx, int ny, int nz)
{
    // delta_m3::extract (injector.cpp:118-140): sum over iy, ix, iz of (yw*xw*zw) u
    ExtTable t;
    t.nrec = op.npts;
    const int nw = op.nw();
    t.gidx.resize((size_t)27 * op.npts);
    t.w.resize((size_t)27 * op.npts);
    for (int r = 0; r < op.npts; r++) {
        const float *xw = &op.xw[(size_t)2 * nw * r + nw], *yw = &op.yw[(size_t)2 * nw * r + nw],
                    *zw = &op.zw[(size_t)2 * nw * r + nw];
        int k = 0;
        for (int iy = 0; iy < 3; iy++)
            for (int ix = 0; ix < 3; ix++)
                for (int iz = 0; iz < 3; iz++, k++) {
                    t.gidx[(size_t)27 * r + k] =
                        ((int64_t)op.yind[3 * r + iy] * nx + op.xind[3 * r + ix]) * nz + op.zind[3 * r + iz];
                    t.w[(size_t)27 * r + k] = yw[iy] * xw[ix] * zw[iz];
                }
    }
    return t;
}

Dipole make_dipole(int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy, float oz,
                   const std::vector<Loc5> &loc, float gl)
{
    // dipole_m3::findIndicesWeights (injector.cpp:313-431): the offsets of
    // the two ends are evaluated in double (cos/sin of float angles), the
    // sub-cell positions stored as float, weights as for delta_m3.
    Dipole d;
    const int npts = (int)loc.size();
    for (PointOp *op : {&d.a, &d.b}) {
        op->npts = npts;
        op->derivative = false;
        op->xind.assign(3 * npts, 0);
        op->yind.assign(3 * npts, 0);
        op->zind.assign(3 * npts, 0);
        op->xw.assign((size_t)6 * npts, 0.f);
        op->yw.assign((size_t)6 * npts, 0.f);
        op->zw.assign((size_t)6 * npts, 0.f);
    }
    auto axis = [&](double pos, float o, float h, int n, int *ind, float *w) {
        int piv = (int)std::round((pos - o) / h);
        if (piv == 0) piv = 1;
        if (piv == n - 1) piv = n - 2;
        ind[0] = piv - 1;
        ind[1] = piv;
        ind[2] = piv + 1;
        const float a = (float)((pos - o) / h - piv);
        const double a2 = std::pow((double)a, 2);
        float *wi = w, *we = w + 3;
        wi[0] = (float)((a2 - a) / (2 * h * hcoef(n, ind[0])));
        wi[1] = (float)((-a2 + 1) / (h * hcoef(n, ind[1])));
        wi[2] = (float)((a2 + a) / (2 * h * hcoef(n, ind[2])));
        we[0] = (float)((a2 - a) / 2);
        we[1] = (float)(-a2 + 1);
        we[2] = (float)((a2 + a) / 2);
    };
    for (int r = 0; r < npts; r++) {
        const Loc5 &l = loc[r];
        const double hx = gl / 2 * std::cos((double)l.dip) * std::cos((double)l.az);
        const double hy = gl / 2 * std::cos((double)l.dip) * std::sin((double)l.az);
        const double hz = gl / 2 * std::sin((double)l.dip);
        axis(l.x - hx, ox, dx, nx, &d.a.xind[3 * r], &d.a.xw[(size_t)6 * r]);
        axis(l.x + hx, ox, dx, nx, &d.b.xind[3 * r], &d.b.xw[(size_t)6 * r]);
        axis(l.y - hy, oy, dy, ny, &d.a.yind[3 * r], &d.a.yw[(size_t)6 * r]);
        axis(l.y + hy, oy, dy, ny, &d.b.yind[3 * r], &d.b.yw[(size_t)6 * r]);
        axis(l.z - hz, oz, dz, nz, &d.a.zind[3 * r], &d.a.zw[(size_t)6 * r]);
        axis(l.z + hz, oz, dz, nz, &d.b.zind[3 * r], &d.b.zw[(size_t)6 * r]);
    }
    return d;
}

ExtTable dipole_extraction_table(const Dipole &d, int nx, int ny, int nz)
{
    // dipole_m3::extract (injector.cpp:467-493): sum of (b weights) u(b) - (a weights) u(a)
    const ExtTable ta = extraction_table(d.a, nx, ny, nz), tb = extraction_table(d.b, nx, ny, nz);
    ExtTable t;
    t.nrec = ta.nrec;
    t.ntap = 54;
    t.gidx.resize((size_t)54 * t.nrec);
    t.w.resize((size_t)54 * t.nrec);
    for (int r = 0; r < t.nrec; r++)
        for (int k = 0; k < 27; k++) {
            t.gidx[(size_t)54 * r + 2 * k] = tb.gidx[(size_t)27 * r + k];
            t.w[(size_t)54 * r + 2 * k] = tb.w[(size_t)27 * r + k];
            t.gidx[(size_t)54 * r + 2 * k + 1] = ta.gidx[(size_t)27 * r + k];
            t.w[(size_t)54 * r + 2 * k + 1] = -ta.w[(size_t)27 * r + k];
        }
    return t;
}

InjTable dipole_injection_table(const Dipole &d, int nx, int ny, int nz, int ncomp_field)
{
    // dipole_m3::inject (injector.cpp:433-465): end a gets -w s, end b +w s
    InjTable ta = injection_table(d.a, nx, ny, nz, ncomp_field), tb = injection_table(d.b, nx, ny, nz, ncomp_field);
    for (int c = 0; c < ncomp_field; c++) {
        for (auto &w : ta.w[c]) w = -w;
        ta.gidx[c].insert(ta.gidx[c].end(), tb.gidx[c].begin(), tb.gidx[c].end());
        ta.trace[c].insert(ta.trace[c].end(), tb.trace[c].begin(), tb.trace[c].end());
        ta.w[c].insert(ta.w[c].end(), tb.w[c].begin(), tb.w[c].end());
    }
    return ta;
}

void dipole_to_strain(bool adj, float *p, const float *dip, const float *az, int nr, int nt, float gl)
{
    float *p0 = p, *p1 = p + (size_t)nr * nt, *p2 = p + 2 * (size_t)nr * nt;
    for (int ix = 0; ix < nr; ix++) {
        const float cd = (float)std::cos((double)dip[ix]), sd = (float)std::sin((double)dip[ix]);
        const float ca = (float)std::cos((double)az[ix]), sa = (float)std::sin((double)az[ix]);
        const size_t o = (size_t)ix * nt;
        for (int it = 0; it < nt; it++) {
            if (!adj) {
                p0[o + it] = (cd * ca * p0[o + it] + cd * sa * p1[o + it] + sd * p2[o + it]) / gl;
                p1[o + it] = 0.f;
                p2[o + it] = 0.f;
            } else {
                p2[o + it] = sd * p0[o + it] / gl;
                p1[o + it] = cd * sa * p0[o + it] / gl;
                p0[o + it] *= cd * ca / gl;
            }
        }
    }
}

bool dipole_inside(const Loc5 &l, float gl, int nx, int ny, int nz, float dx, float dy, float dz, float ox, float oy,
                   float oz)
{
    const double hx = gl / 2 * std::cos((double)l.dip) * std::cos((double)l.az);
    const double hy = gl / 2 * std::cos((double)l.dip) * std::sin((double)l.az);
    const double hz = gl / 2 * std::sin((double)l.dip);
    auto in = [](double v, float o, float d, int n) { return !(v < o || v > o + (n - 1) * d); };
    return in(l.x - hx, ox, dx, nx) && in(l.x + hx, ox, dx, nx) && in(l.y - hy, oy, dy, ny) &&
           in(l.y + hy, oy, dy, ny) && in(l.z - hz, oz, dz, nz) && in(l.z + hz, oz, dz, nz);
}

void apply_h3(float *g, int nx, int ny, int nz, float dx, float dy, float dz)
{
    // applyHx, applyHy, applyHz in that order (we_op.cpp:1033-1038; spatial_operators.cpp:11-177)
    for (int iy = 0; iy < ny; iy++)
        for (int ix = 0; ix < nx; ix++) {
            const float cx = (ix < 4) ? kH[ix] : (ix >= nx - 4 ? kH[nx - 1 - ix] : 0.f);
            float *p = g + ((int64_t)iy * nx + ix) * nz;
            for (int iz = 0; iz < nz; iz++) p[iz] = cx != 0.f ? p[iz] * cx * dx : p[iz] * dx;
        }
    for (int iy = 0; iy < ny; iy++) {
        const float cy = (iy < 4) ? kH[iy] : (iy >= ny - 4 ? kH[ny - 1 - iy] : 0.f);
        float *p = g + (int64_t)iy * nx * nz;
        for (int64_t i = 0; i < (int64_t)nx * nz; i++) p[i] = cy != 0.f ? p[i] * cy * dy : p[i] * dy;
    }
    for (int64_t c = 0; c < (int64_t)nx * ny; c++) {
        float *p = g + c * nz;
        for (int iz = 0; iz < nz; iz++) {
            const float cz = (iz < 4) ? kH[iz] : (iz >= nz - 4 ? kH[nz - 1 - iz] : 0.f);
            p[iz] = cz != 0.f ? p[iz] * cz * dz : p[iz] * dz;
        }
    }
}

void gradient_to_velocity(float *g, const float *m, int nmodels, int64_t n)
{
    float *g0 = g, *g1 = g + n, *g2 = g + 2 * n;
    const float *p0 = m, *p1 = m + n, *p2 = m + 2 * n;
    if (nmodels >= 3) {
        // we_op.cpp:1049-1058
        for (int64_t i = 0; i < n; i++) {
            g2[i] = (p0[i] / p2[i]) * g0[i] + (p1[i] / p2[i]) * g1[i] + g2[i];
            g1[i] = (float)(2 * std::sqrt((double)(p1[i] * p2[i])) * (g1[i] - 2 * g0[i]));
            g0[i] = (float)(2 * std::sqrt((double)(p2[i] * (p0[i] + 2 * p1[i]))) * g0[i]);
        }
    } else {
        // we_op.cpp:1061-1066
        for (int64_t i = 0; i < n; i++) {
            g1[i] = p1[i] * p0[i] * g0[i] - p1[i] * p1[i] * g1[i];
            g0[i] = (float)(2 * std::sqrt((double)(p0[i] / p1[i])) * g0[i]);
        }
    }
}

// ---------------------------------------------------------------------------
// Absorbing-boundary divisors
// ---------------------------------------------------------------------------
namespace {

struct DivCtx {
    const float *m;
    int nmodels, nx, ny, nz;
    float d[3];  // dx, dy, dz indexed by axis (0 x, 1 y, 2 z)
    float dt, h0;
    const int *bc;
    int64_t idx(int ix, int iy, int iz) const { return ((int64_t)iy * nx + ix) * nz + iz; }
    bool abs(int face) const { return bc[face] == 2; }
};

// Elastic material ratio G(n, c) at point i: mu/rho off-axis, (lambda+2mu)/rho on
// the normal axis, scaled by (1+2eps) on x/y faces of VTI when `aniso` is set.
inline float elastic_ratio(const DivCtx &c, int64_t i, int n, int comp, bool aniso)
{
    const int64_t N = (int64_t)c.nx * c.ny * c.nz;
    const float lam = c.m[i], mu = c.m[N + i], rho = c.m[2 * N + i];
    if (comp != n) return mu / rho;
    float f = 1.f;
    if (aniso && n != 2 && c.nmodels == 6) f = 1 + 2 * c.m[4 * N + i];
    if (aniso) return f * (lam + 2 * mu) / rho;
    return (lam + 2 * mu) / rho;
}

// One face term sqrt(G) dt / (2 d_n h0) in double.
inline double eterm(const DivCtx &c, int64_t i, int n, int comp, bool aniso)
{
    return std::sqrt((double)elastic_ratio(c, i, n, comp, aniso)) * c.dt / (double)(2 * c.d[n] * c.h0);
}

inline double aterm(const DivCtx &c, int64_t i, int n)
{
    const int64_t N = (int64_t)c.nx * c.ny * c.nz;
    return std::sqrt((double)(c.m[i] * c.m[N + i])) * c.dt / (double)(2 * c.d[n] * c.h0);
}

// Acoustic two-face edge term sqrt(K b) dt (da+db) / (2 da db h0)
// (spatial_operators.cpp:653, 845).
inline double aterm2(const DivCtx &c, int64_t i, int na, int nb)
{
    const int64_t N = (int64_t)c.nx * c.ny * c.nz;
    return std::sqrt((double)(c.m[i] * c.m[N + i])) * c.dt * (double)(c.d[na] + c.d[nb]) /
           (double)(2 * c.d[na] * c.d[nb] * c.h0);
}

}  // namespace

ScaleTables boundary_divisors(const float *m, int nmodels, int nx, int ny, int nz, float dx, float dy, float dz,
                              float dt, const int bc[6])
{
    ScaleTables T;
    const int ncomp = nmodels == 2 ? 1 : 3;
    const int64_t fsz[6] = {(int64_t)ny * nx, (int64_t)ny * nx, (int64_t)ny * nz,
                            (int64_t)ny * nz, (int64_t)nx * nz, (int64_t)nx * nz};
    for (int f = 0; f < 6; f++)
        for (int c = 0; c < ncomp; c++) T.f[f][c].assign(fsz[f], 1.f);

    DivCtx C{m, nmodels, nx, ny, nz, {dx, dy, dz}, dt, (float)(17.0 / 48), bc};
    // face (normal axis, side) -> index; axis 0 x, 1 y, 2 z
    auto face_of = [](int n, int hi) { return n == 2 ? (hi ? 1 : 0) : (n == 0 ? (hi ? 3 : 2) : (hi ? 5 : 4)); };
    // divisor storage of a point on its owning face
    auto slot = [&](int ix, int iy, int iz, int c) -> float & {
        if (iz == 0) return T.f[0][c][(int64_t)iy * nx + ix];
        if (iz == nz - 1) return T.f[1][c][(int64_t)iy * nx + ix];
        if (ix == 0) return T.f[2][c][(int64_t)iy * nz + iz];
        if (ix == nx - 1) return T.f[3][c][(int64_t)iy * nz + iz];
        if (iy == 0) return T.f[4][c][(int64_t)ix * nz + iz];
        return T.f[5][c][(int64_t)ix * nz + iz];
    };
    auto put = [&](int ix, int iy, int iz, int c, double s) { slot(ix, iy, iz, c) = 1 + (float)s; };

    // Single-face scaler on face with normal n (edges not shared with another
    // absorbing face are treated with it), and the combined edge scaler.
    auto single = [&](int64_t i, int n, int comp) -> double {
        if (nmodels == 2) return aterm(C, i, n);
        return eterm(C, i, n, comp, true);
    };
    auto pair = [&](int64_t i, int na, int nb, int comp) -> double {
        if (nmodels == 2) return aterm2(C, i, na, nb);
        return eterm(C, i, na, comp, true) + eterm(C, i, nb, comp, true);
    };

    // z faces own their face interior and the four edges at that depth.
    for (int hi = 0; hi < 2; hi++) {
        if (!C.abs(face_of(2, hi))) continue;
        const int iz = hi ? nz - 1 : 0;
        for (int iy = 1; iy < ny - 1; iy++)
            for (int ix = 1; ix < nx - 1; ix++)
                for (int c = 0; c < ncomp; c++) put(ix, iy, iz, c, single(C.idx(ix, iy, iz), 2, c));
        for (int side = 0; side < 2; side++) {
            const int ix = side ? nx - 1 : 0;
            const bool other = C.abs(face_of(0, side));
            for (int iy = 1; iy < ny - 1; iy++)
                for (int c = 0; c < ncomp; c++) {
                    const int64_t i = C.idx(ix, iy, iz);
                    put(ix, iy, iz, c, other ? pair(i, 2, 0, c) : single(i, 2, c));
                }
        }
        for (int side = 0; side < 2; side++) {
            const int iy = side ? ny - 1 : 0;
            const bool other = C.abs(face_of(1, side));
            for (int ix = 1; ix < nx - 1; ix++)
                for (int c = 0; c < ncomp; c++) {
                    const int64_t i = C.idx(ix, iy, iz);
                    put(ix, iy, iz, c, other ? pair(i, 2, 1, c) : single(i, 2, c));
                }
        }
    }
    // x faces: interior, z edges when the z face is not absorbing, y edges shared.
    for (int hi = 0; hi < 2; hi++) {
        if (!C.abs(face_of(0, hi))) continue;
        const int ix = hi ? nx - 1 : 0;
        for (int iy = 1; iy < ny - 1; iy++)
            for (int iz = 1; iz < nz - 1; iz++)
                for (int c = 0; c < ncomp; c++) put(ix, iy, iz, c, single(C.idx(ix, iy, iz), 0, c));
        for (int side = 0; side < 2; side++) {
            if (C.abs(face_of(2, side))) continue;
            const int iz = side ? nz - 1 : 0;
            for (int iy = 1; iy < ny - 1; iy++)
                for (int c = 0; c < ncomp; c++) put(ix, iy, iz, c, single(C.idx(ix, iy, iz), 0, c));
        }
        for (int side = 0; side < 2; side++) {
            const int iy = side ? ny - 1 : 0;
            const bool other = C.abs(face_of(1, side));
            for (int iz = 1; iz < nz - 1; iz++)
                for (int c = 0; c < ncomp; c++) {
                    const int64_t i = C.idx(ix, iy, iz);
                    put(ix, iy, iz, c, other ? pair(i, 0, 1, c) : single(i, 0, c));
                }
        }
    }
    // y faces: interior and the edges no other absorbing face took.
    for (int hi = 0; hi < 2; hi++) {
        if (!C.abs(face_of(1, hi))) continue;
        const int iy = hi ? ny - 1 : 0;
        for (int ix = 1; ix < nx - 1; ix++)
            for (int iz = 1; iz < nz - 1; iz++)
                for (int c = 0; c < ncomp; c++) put(ix, iy, iz, c, single(C.idx(ix, iy, iz), 1, c));
        for (int side = 0; side < 2; side++) {
            if (C.abs(face_of(2, side))) continue;
            const int iz = side ? nz - 1 : 0;
            for (int ix = 1; ix < nx - 1; ix++)
                for (int c = 0; c < ncomp; c++) put(ix, iy, iz, c, single(C.idx(ix, iy, iz), 1, c));
        }
        for (int side = 0; side < 2; side++) {
            if (C.abs(face_of(0, side))) continue;
            const int ix = side ? nx - 1 : 0;
            for (int iz = 1; iz < nz - 1; iz++)
                for (int c = 0; c < ncomp; c++) put(ix, iy, iz, c, single(C.idx(ix, iy, iz), 1, c));
        }
    }
    // Corners: each absorbing face adds its single term (isotropic ratio, no
    // (1+2eps)) into a float accumulator, faces in the order top, bottom, left,
    // right, front, back (spatial_operators.hpp:1885-2567).
    const int cx[8] = {0, nx - 1, nx - 1, 0, 0, nx - 1, nx - 1, 0};
    const int cy[8] = {0, 0, ny - 1, ny - 1, 0, 0, ny - 1, ny - 1};
    const int cz[8] = {0, 0, 0, 0, nz - 1, nz - 1, nz - 1, nz - 1};
    for (int k = 0; k < 8; k++) {
        const int64_t i = C.idx(cx[k], cy[k], cz[k]);
        for (int c = 0; c < ncomp; c++) {
            float psc = 0.f;
            const int faces[6] = {0, 1, 2, 3, 4, 5};
            for (int fi = 0; fi < 6; fi++) {
                const int f = faces[fi];
                if (!C.abs(f)) continue;
                const int n = f < 2 ? 2 : (f < 4 ? 0 : 1);
                const int hi = f & 1;
                const bool on = (n == 2 && cz[k] == (hi ? nz - 1 : 0)) || (n == 0 && cx[k] == (hi ? nx - 1 : 0)) ||
                                (n == 1 && cy[k] == (hi ? ny - 1 : 0));
                if (!on) continue;
                const double term = nmodels == 2 ? aterm(C, i, n) : eterm(C, i, n, c, false);
                psc = (float)((double)psc + term);
            }
            slot(cx[k], cy[k], cz[k], c) = 1 + psc;
        }
    }
    return T;
}

TaperTables taper_tables(int nx, int ny, int nz, const int taper[6], float a)
{
    // taperz/x/y (spatial_operators.cpp:408-506): lo side (izmin = T, izmax = 0)
    // val = cos(a pi/2 (i+1-T)/(-T)); hi side (izmin = n-T, izmax = n)
    // val = cos(a pi/2 (i-(n-T))/T); factor val*val in float.
    TaperTables t;
    const int n[3] = {nz, nx, ny};
    for (int ax = 0; ax < 3; ax++) {
        std::vector<float> &lo = t.t[2 * ax], &hi = t.t[2 * ax + 1];
        lo.assign(n[ax], 1.f);
        hi.assign(n[ax], 1.f);
        const int Tlo = taper[ax == 0 ? 0 : (ax == 1 ? 2 : 4)];
        const int Thi = taper[ax == 0 ? 1 : (ax == 1 ? 3 : 5)];
        if (Tlo > 0)
            for (int i = 0; i < Tlo && i < n[ax]; i++) {
                const float v = (float)std::cos(a * 0.5 * M_PI * (i + 1 - Tlo) / (0 - Tlo));
                lo[i] = v * v;
            }
        if (Thi > 0) {
            const int i0 = n[ax] - Thi;
            for (int i = std::max(0, i0); i < n[ax]; i++) {
                const float v = (float)std::cos(a * 0.5 * M_PI * (i - i0) / (n[ax] - i0));
                hi[i] = v * v;
            }
        }
    }
    return t;
}

}  // namespace fwi
