// Host float64 cosmology: E(a), growth ODE tables, superconformal time, the
// timetable lookups and the per-step coefficients of the three steppers.
//
// Same algorithm as native/DiscoDJNative/src/cosmology/Cosmology.jl:47-115,
// src/cosmology/growth.jl:23-96, src/nbody/timetables.jl:10-45 and
// src/nbody/run_nbody.jl:22-101 (kept alike because the coefficients must agree
// with the reference's to round-off: same table grid, same RK4 in ln a, same
// `jnp.interp` lookups, same Gauss-Legendre rule).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "common.h"

namespace djb {

static thread_local std::string g_err;

void set_error(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
}

void clear_error() { g_err.clear(); }

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

const char* last_error() { return g_err.c_str(); }

}  // namespace djb

struct djb_cosmology {
    double Omega_c, Omega_b, h, sigma8, n_s, Omega_k, w0, wa;
    std::vector<double> a, D1, D2, D3a, D3b, D3c, f1, f2, f3a, f3b, sct;
    std::vector<double> Dda, D2da;  // f1*D1/a, f2*D2/a
    double D1_at1;

    double Om() const { return Omega_c + Omega_b; }
    double Ode(double x) const {
        return (1.0 - Om() - Omega_k) * std::pow(x, -3.0 * (1.0 + w0 + wa)) *
               std::exp(-3.0 * wa * (1.0 - x));
    }
    double E(double x) const {
        return std::sqrt(Om() * std::pow(x, -3.0) + Omega_k * std::pow(x, -2.0) + Ode(x));
    }
};

namespace {

using djb::fail;

// growth.jl:23-45; y = [ln D1, f1, ln|D2|, f2, ln D3a, f3a, ln|D3b|, f3b, ln D3c]
void growth_derivs(const djb_cosmology& c, double lna, const double* y, double* dy) {
    const double a = std::exp(lna);
    const double e = c.E(a);
    const double Esq = e * e;
    const double Om_a = (c.Om() * std::pow(a, -3.0)) / Esq;
    const double Ox_a = c.Ode(a) / Esq;
    const double w_a = c.w0 + c.wa * (1.0 - a);
    const double drag = 1.0 - 0.5 * (Om_a + (1.0 + 3.0 * w_a) * Ox_a);
    const double y1 = y[0], f1 = y[1], y2 = y[2], f2 = y[3], y3a = y[4], f3a = y[5];
    const double y3b = y[6], f3b = y[7], y3c = y[8];
    const double D1 = std::exp(y1), D1sq = D1 * D1, D1cu = D1sq * D1;
    const double D2 = -std::exp(y2), D3a = std::exp(y3a), D3b = -std::exp(y3b);
    const double D3c = std::exp(y3c);
    dy[0] = f1;
    dy[1] = 1.5 * Om_a - f1 * f1 - f1 * drag;
    dy[2] = f2;
    dy[3] = 1.5 * Om_a * (1.0 - D1sq / D2) - f2 * f2 - f2 * drag;
    dy[4] = f3a;
    dy[5] = 1.5 * Om_a * (1.0 + 2.0 * D1cu / D3a) - f3a * f3a - f3a * drag;
    dy[6] = f3b;
    dy[7] = 1.5 * Om_a * (1.0 + (2.0 * D1 * D2 - 2.0 * D1cu) / D3b) - f3b * f3b - f3b * drag;
    dy[8] = D1 * D2 / D3c * (f1 - f2);
}

void rk4_growth(const djb_cosmology& c, double lna, double* y, double dl) {
    double k1[9], k2[9], k3[9], k4[9], t[9];
    growth_derivs(c, lna, y, k1);
    for (int i = 0; i < 9; ++i) t[i] = y[i] + dl / 2 * k1[i];
    growth_derivs(c, lna + dl / 2, t, k2);
    for (int i = 0; i < 9; ++i) t[i] = y[i] + dl / 2 * k2[i];
    growth_derivs(c, lna + dl / 2, t, k3);
    for (int i = 0; i < 9; ++i) t[i] = y[i] + dl * k3[i];
    growth_derivs(c, lna + dl, t, k4);
    for (int i = 0; i < 9; ++i) y[i] = y[i] + dl / 6 * (k1[i] + 2 * k2[i] + 2 * k3[i] + k4[i]);
}

// Julia LinRange element j of n: (1 - t) a + t b, t = j/(n-1).
double linrange(double a, double b, int j, int n) {
    if (j == 0) return a;
    if (j == n - 1) return b;
    const double t = double(j) / double(n - 1);
    return (1.0 - t) * a + t * b;
}

// timetables.jl:10-18 (`jnp.interp`: clamp outside; xp ascending)
double jinterp(double x, const std::vector<double>& xp, const std::vector<double>& fp) {
    const size_t n = xp.size();
    if (x <= xp[0]) return fp[0];
    if (x >= xp[n - 1]) return fp[n - 1];
    size_t i = size_t(std::upper_bound(xp.begin(), xp.end(), x) - xp.begin()) - 1;
    if (i >= n - 1) return fp[n - 1];
    const double t = (x - xp[i]) / (xp[i + 1] - xp[i]);
    return fp[i] + t * (fp[i + 1] - fp[i]);
}

void build_tables(djb_cosmology& c, int n, double a_ini) {
    c.a.resize(n);
    const double l0 = std::log10(a_ini);
    for (int j = 0; j < n; ++j) c.a[j] = std::pow(10.0, linrange(l0, 0.0, j, n));
    std::vector<double> Y(9 * size_t(n));
    const double amin = c.a[0];
    double y[9] = {std::log(amin), 1.0, std::log(3.0 / 7.0 * amin * amin), 2.0,
                   std::log(1.0 / 3.0 * amin * amin * amin), 3.0,
                   std::log(10.0 / 21.0 * amin * amin * amin), 3.0,
                   std::log(1.0 / 7.0 * amin * amin * amin)};
    std::memcpy(&Y[0], y, sizeof y);
    for (int i = 1; i < n; ++i) {
        const double l_prev = std::log(c.a[i - 1]);
        rk4_growth(c, l_prev, y, std::log(c.a[i]) - l_prev);
        std::memcpy(&Y[9 * size_t(i)], y, sizeof y);
    }
    auto col = [&](int k) {
        std::vector<double> v(n);
        for (int i = 0; i < n; ++i) v[i] = Y[9 * size_t(i) + k];
        return v;
    };
    std::vector<double> l1 = col(0), l2 = col(2), l3a = col(4), l3b = col(6), l3c = col(8);
    c.f1 = col(1);
    c.f2 = col(3);
    c.f3a = col(5);
    c.f3b = col(7);
    c.D1.resize(n);
    c.D2.resize(n);
    c.D3a.resize(n);
    c.D3b.resize(n);
    c.D3c.resize(n);
    for (int i = 0; i < n; ++i) c.D1[i] = std::exp(l1[i]);
    // LinearInterpolation(a, D1)(1.0): a[end] == 1 exactly
    c.D1_at1 = jinterp(1.0, c.a, c.D1);
    const double d1 = c.D1_at1, d2 = d1 * d1, d3 = d2 * d1;
    for (int i = 0; i < n; ++i) {
        c.D1[i] = c.D1[i] / d1;
        c.D2[i] = -std::exp(l2[i]) / d2;
        c.D3a[i] = std::exp(l3a[i]) / d3;
        c.D3b[i] = -std::exp(l3b[i]) / d3;
        c.D3c[i] = std::exp(l3c[i]) / d3;
    }
    // growth.jl:88-96
    std::vector<double> f(n);
    for (int i = 0; i < n; ++i) f[i] = 1.0 / (c.E(c.a[i]) * c.a[i] * c.a[i] * c.a[i]);
    c.sct.assign(n, 0.0);
    for (int i = n - 2; i >= 0; --i)
        c.sct[i] = c.sct[i + 1] - (c.a[i + 1] - c.a[i]) * (f[i] + f[i + 1]) / 2;
    const double last = c.sct[n - 1];
    for (int i = 0; i < n; ++i) c.sct[i] -= last;
    c.Dda.resize(n);
    c.D2da.resize(n);
    for (int i = 0; i < n; ++i) {
        c.Dda[i] = c.f1[i] * c.D1[i] / c.a[i];
        c.D2da[i] = c.f2[i] * c.D2[i] / c.a[i];
    }
}

double Dplus(const djb_cosmology& c, double a) { return jinterp(a, c.a, c.D1); }
double Dplusda(const djb_cosmology& c, double a) { return jinterp(a, c.a, c.Dda); }
double D2plus(const djb_cosmology& c, double a) { return jinterp(a, c.a, c.D2); }
double D2plusda(const djb_cosmology& c, double a) { return jinterp(a, c.a, c.D2da); }
double superconft(const djb_cosmology& c, double a) { return jinterp(a, c.a, c.sct); }
double a_of_superconft(const djb_cosmology& c, double s) { return jinterp(s, c.sct, c.a); }
double a_of_Dplus(const djb_cosmology& c, double D) { return jinterp(D, c.D1, c.a); }
double Fplus(const djb_cosmology& c, double a) { return a * a * a * c.E(a) * Dplusda(c, a); }

// run_nbody.jl:22 (numpy.linspace)
std::vector<double> nplinspace(double s, double e, int num) {
    std::vector<double> y(num);
    const double st = (e - s) / (num - 1);
    for (int i = 0; i < num; ++i) y[i] = s + i * st;
    y[num - 1] = e;
    return y;
}

const double GL5_X[5] = {-0.906179845938664, -0.5384693101056831, 0.0, 0.5384693101056831,
                         0.906179845938664};
const double GL5_W[5] = {0.23692688505618928, 0.4786286704993663, 0.5688888888888887,
                         0.4786286704993663, 0.23692688505618928};

}  // namespace

extern "C" {

const char* djb_last_error(void) { return djb::last_error(); }

int djb_cosmology_create(const double p[8], int32_t n_pts, double a_ini, djb_cosmology** out) {
    djb::clear_error();
    if (!p || !out) return fail(DJB_ERR_INVALID, "djb_cosmology_create: null argument");
    if (n_pts < 2) return fail(DJB_ERR_INVALID, "n_pts must be >= 2");
    if (!(a_ini > 0.0 && a_ini < 1.0)) return fail(DJB_ERR_INVALID, "a_ini must be in (0, 1)");
    djb_cosmology* c = new (std::nothrow) djb_cosmology();
    if (!c) return fail(DJB_ERR_ALLOC, "host allocation failed");
    c->Omega_c = p[0];
    c->Omega_b = p[1];
    c->h = p[2];
    c->sigma8 = p[3];
    c->n_s = p[4];
    c->Omega_k = p[5];
    c->w0 = p[6];
    c->wa = p[7];
    try {
        build_tables(*c, n_pts, a_ini);
    } catch (...) {
        delete c;
        return fail(DJB_ERR_ALLOC, "host allocation failed");
    }
    *out = c;
    return DJB_OK;
}

int djb_cosmology_create_named(const char* name, djb_cosmology** out) {
    djb::clear_error();
    // Cosmology.jl:145-150
    struct Named {
        const char* name;
        double p[8];
    };
    static const Named table[] = {
        {"Planck18EEBAOSN", {0.259622, 0.0488911, 0.67742, 0.8105, 0.96822, 0.0, -1.0, 0.0}},
        {"Planck15", {0.2589, 0.0486, 0.6774, 0.8159, 0.9667, 0.0, -1.0, 0.0}},
        {"Quijote", {0.3175, 0.049, 0.6711, 0.834, 0.9624, 0.0, -1.0, 0.0}},
        {"CamelsCV", {0.2514, 0.049, 0.6711, 0.818, 0.9624, 0.0, -1.0, 0.0}},
    };
    if (!name) return fail(DJB_ERR_INVALID, "null cosmology name");
    for (const Named& t : table)
        if (std::strcmp(t.name, name) == 0) return djb_cosmology_create(t.p, 2500, 1e-10, out);
    return fail(DJB_ERR_INVALID,
                "Unknown cosmology: %s. Available: Planck18EEBAOSN, Planck15, Quijote, CamelsCV",
                name);
}

int djb_cosmology_destroy(djb_cosmology* c) {
    delete c;
    return DJB_OK;
}

int djb_cosmology_table_size(const djb_cosmology* c, int32_t* n) {
    if (!c || !n) return fail(DJB_ERR_INVALID, "null argument");
    *n = int32_t(c->a.size());
    return DJB_OK;
}

int djb_cosmology_table(const djb_cosmology* c, int32_t which, double* out, int32_t n) {
    djb::clear_error();
    if (!c || !out) return fail(DJB_ERR_INVALID, "null argument");
    if (size_t(n) != c->a.size()) return fail(DJB_ERR_INVALID, "table length mismatch");
    const std::vector<double>* v = nullptr;
    switch (which) {
        case 0: v = &c->a; break;
        case 1: v = &c->D1; break;
        case 2: v = &c->Dda; break;
        case 3: v = &c->D2; break;
        case 4: v = &c->D2da; break;
        case 5: v = &c->sct; break;
        case 6: v = &c->f1; break;
        case 7: v = &c->f2; break;
        case 8: v = &c->D3a; break;
        case 9: v = &c->D3b; break;
        case 10: v = &c->D3c; break;
        default: return fail(DJB_ERR_INVALID, "unknown table %d", which);
    }
    std::memcpy(out, v->data(), sizeof(double) * v->size());
    return DJB_OK;
}

int djb_cosmology_params(const djb_cosmology* c, double out[8]) {
    if (!c || !out) return fail(DJB_ERR_INVALID, "null argument");
    const double p[8] = {c->Omega_c, c->Omega_b, c->h, c->sigma8, c->n_s, c->Omega_k, c->w0, c->wa};
    std::memcpy(out, p, sizeof p);
    return DJB_OK;
}

int djb_cosmology_d1_unnormed(const djb_cosmology* c, double* out) {
    if (!c || !out) return fail(DJB_ERR_INVALID, "null argument");
    *out = c->D1_at1;
    return DJB_OK;
}

int djb_cosmology_eval(const djb_cosmology* c, int32_t what, double x, double* out) {
    djb::clear_error();
    if (!c || !out) return fail(DJB_ERR_INVALID, "null argument");
    switch (what) {
        case 0: *out = Dplus(*c, x); break;
        case 1: *out = Dplusda(*c, x); break;
        case 2: *out = D2plus(*c, x); break;
        case 3: *out = D2plusda(*c, x); break;
        case 4: *out = superconft(*c, x); break;
        case 5: *out = a_of_superconft(*c, x); break;
        case 6: *out = a_of_Dplus(*c, x); break;
        case 7: *out = Fplus(*c, x); break;
        case 8: *out = c->E(x); break;
        case 9: *out = c->Om(); break;
        default: return fail(DJB_ERR_INVALID, "unknown quantity %d", what);
    }
    return DJB_OK;
}

int djb_stepper_coefficients(const djb_cosmology* c, int32_t stepper, int32_t time_var,
                             const double* tv_array, double a_ini, double a_end, int32_t n_steps,
                             double* alpha, double* beta, double* dd1, double* dd2,
                             double* all_a_out) {
    djb::clear_error();
    if (!c || !alpha || !beta || !dd1 || !dd2 || !all_a_out)
        return fail(DJB_ERR_INVALID, "null argument");
    if (n_steps < 1) return fail(DJB_ERR_INVALID, "n_steps must be >= 1");
    const int ns = n_steps;
    std::vector<double> all_int;
    std::function<double(double)> itoa;
    std::vector<double> tgrid, tvv;
    if (time_var == DJB_TIME_ARRAY) {
        if (!tv_array) return fail(DJB_ERR_INVALID, "time_var vector must have n_steps + 1 entries");
        tvv.assign(tv_array, tv_array + ns + 1);
        tgrid = nplinspace(0.0, double(ns), ns + 1);
        itoa = [&](double x) { return jinterp(x, tgrid, tvv); };
        all_int = nplinspace(0.0, double(ns), ns + 1);
    } else {
        std::function<double(double)> a2i;
        switch (time_var) {
            case DJB_TIME_A:
                a2i = [](double a) { return a; };
                itoa = [](double x) { return x; };
                break;
            case DJB_TIME_LOG_A:
                a2i = [](double a) { return std::log(a); };
                itoa = [](double x) { return std::exp(x); };
                break;
            case DJB_TIME_D:
                a2i = [&](double a) { return Dplus(*c, a); };
                itoa = [&](double x) { return a_of_Dplus(*c, x); };
                break;
            case DJB_TIME_SUPERCONFT:
                a2i = [&](double a) { return superconft(*c, a); };
                itoa = [&](double x) { return a_of_superconft(*c, x); };
                break;
            default:
                return fail(DJB_ERR_INVALID,
                            "time_var must be :a, :log_a, :D, :superconft or a vector of scale factors");
        }
        all_int = nplinspace(a2i(a_ini), a2i(a_end), ns + 1);
    }
    std::vector<double> all_a(ns + 1), a_mid(ns);
    for (int i = 0; i <= ns; ++i) all_a[i] = itoa(all_int[i]);
    for (int i = 0; i < ns; ++i) a_mid[i] = itoa((all_int[i] + all_int[i + 1]) / 2);
    if (stepper == DJB_STEPPER_BULLFROG) {
        const double D1 = c->D1_at1;
        for (int i = 0; i < ns; ++i) {
            const double ab = all_a[i], ae = all_a[i + 1];
            const double D_b = Dplus(*c, ab) * D1, D_e = Dplus(*c, ae) * D1;
            const double Dda_b = Dplusda(*c, ab) * D1, Dda_e = Dplusda(*c, ae) * D1;
            const double D2_b = D2plus(*c, ab) * (D1 * D1);
            const double D2da_b = D2plusda(*c, ab) * (D1 * D1);
            const double D2da_e = D2plusda(*c, ae) * (D1 * D1);
            const double dD = D_e - D_b;
            const double xi = D_b / dD;
            const double bracket =
                (D2_b + D2da_b / Dda_b * dD / 2) / ((xi + 0.5) * dD) - (xi + 0.5) * dD;
            alpha[i] = (D2da_e / Dda_e - bracket) / (D2da_b / Dda_b - bracket);
            const double D_mid = Dplus(*c, a_mid[i]);
            beta[i] = (1 - alpha[i]) / D_mid;
            dd1[i] = D_mid - D_b / D1;
            dd2[i] = D_e / D1 - D_mid;
        }
    } else if (stepper == DJB_STEPPER_FASTPM) {
        for (int i = 0; i < ns; ++i) {
            alpha[i] = Fplus(*c, all_a[i]) / Fplus(*c, all_a[i + 1]);
            const double D_mid = Dplus(*c, a_mid[i]);
            beta[i] = (1 - alpha[i]) / D_mid;
            dd1[i] = D_mid - Dplus(*c, all_a[i]);
            dd2[i] = Dplus(*c, all_a[i + 1]) - D_mid;
        }
    } else if (stepper == DJB_STEPPER_SYMPLECTIC) {
        auto f = [&](double a) { return 1.0 / (a * a * c->E(a)); };
        for (int i = 0; i < ns; ++i) {
            const double b = all_a[i], e = all_a[i + 1];
            double s = 0.0;
            for (int j = 0; j < 5; ++j) s += GL5_W[j] * f(0.5 * (e - b) * GL5_X[j] + 0.5 * (b + e));
            alpha[i] = 1.0;
            beta[i] = 1.5 * c->Om() * (0.5 * (e - b) * s);
            const double scm = superconft(*c, a_mid[i]);
            dd1[i] = scm - superconft(*c, b);
            dd2[i] = superconft(*c, e) - scm;
        }
    } else {
        return fail(DJB_ERR_INVALID, "stepper must be :bullfrog, :fastpm or :symplectic");
    }
    std::memcpy(all_a_out, all_a.data(), sizeof(double) * (ns + 1));
    return DJB_OK;
}

}  // extern "C"
