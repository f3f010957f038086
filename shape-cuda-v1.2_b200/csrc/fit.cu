// bestfit driver of the SHAPE B200 engine: one-parameter-at-a-time line
// minimisations of the objective (src/shape/bestfit.c:250-704), every trial
// evaluated on the device (a CUDA-graph replay for the batched forms).
//
// The two line searches are written from their published descriptions:
//  - bracketing by golden-ratio expansion with parabolic extrapolation
//    (the bracketing step used before Brent's method in the reference,
//    src/nr/mnbrak.c), growth factor 1.618034, extrapolation limit 100,
//    denominator floor 1e-20;
//  - Brent's minimiser (R. P. Brent, Algorithms for Minimization without
//    Derivatives, 1973, procedure localmin) with the reference's absolute
//    tolerance extension: the acceptance tolerance is tol*|x| + max(abstol,
//    1e-10) (src/nr/brent_abs.c), golden section 0.3819660, at most 100
//    iterations.
// The decision steps and constants are kept identical so that, given the
// same objective values, the sequence of trial parameter values matches the
// reference's exactly (pinned by tests/test_linesearch.py).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "shape_b200.h"

namespace shape {
int report_error(int code, const std::string &msg);

namespace {

// SIGN(a, b) of the reference's numerical helpers: |a| when b > 0, else -|a|
inline double signed_mag(double a, double b) { return (b > 0.0) ? fabs(a) : -fabs(a); }

struct Bracket {
    double a, b, c, fa, fb, fc;
};

template <class F>
void bracket_minimum(F &f, Bracket &br)
{
    const double grow = 1.618034, limit = 100.0, tiny = 1.0e-20;
    br.fa = f(br.a);
    br.fb = f(br.b);
    if (br.fb > br.fa) {                    // walk downhill from a to b
        double t = br.a; br.a = br.b; br.b = t;
        t = br.fa; br.fa = br.fb; br.fb = t;
    }
    br.c = br.b + grow * (br.b - br.a);
    br.fc = f(br.c);
    while (br.fb > br.fc) {
        // parabola through (a, fa), (b, fb), (c, fc): its vertex u
        const double r = (br.b - br.a) * (br.fb - br.fc);
        const double q = (br.b - br.c) * (br.fb - br.fa);
        double u = br.b - ((br.b - br.c) * q - (br.b - br.a) * r) /
                              (2.0 * signed_mag(std::max(fabs(q - r), tiny), q - r));
        const double ulim = br.b + limit * (br.c - br.b);
        double fu;
        if ((br.b - u) * (u - br.c) > 0.0) {            // vertex between b and c
            fu = f(u);
            if (fu < br.fc) {                           // minimum between b and c
                br.a = br.b; br.b = u; br.fa = br.fb; br.fb = fu;
                return;
            }
            if (fu > br.fb) {                           // minimum between a and u
                br.c = u; br.fc = fu;
                return;
            }
            u = br.c + grow * (br.c - br.b);            // parabola useless: grow
            fu = f(u);
        } else if ((br.c - u) * (u - ulim) > 0.0) {     // vertex between c and the limit
            fu = f(u);
            if (fu < br.fc) {
                br.b = br.c; br.c = u; u = br.c + grow * (br.c - br.b);
                br.fb = br.fc; br.fc = fu; fu = f(u);
            }
        } else if ((u - ulim) * (ulim - br.c) >= 0.0) { // vertex beyond the limit
            u = ulim;
            fu = f(u);
        } else {                                        // vertex on the wrong side
            u = br.c + grow * (br.c - br.b);
            fu = f(u);
        }
        br.a = br.b; br.b = br.c; br.c = u;
        br.fa = br.fb; br.fb = br.fc; br.fc = fu;
    }
}

// Returns the minimum value; *iters_out = -1 when 100 iterations did not
// meet the tolerance (the reference reports this and exits).
template <class F>
double brent_minimize(F &f, double ax, double bx, double cx, double tol, double abstol,
                      double *xmin, int *iters_out)
{
    const int maxit = 100;
    const double cgold = 0.3819660, zeps = 1.0e-10;
    const double abst = (abstol > zeps) ? abstol : zeps;
    double a = (ax < cx) ? ax : cx, b = (ax > cx) ? ax : cx;
    double x = bx, w = bx, v = bx;
    double fx = f(x), fw = fx, fv = fx;
    double d = 0.0, e = 0.0;
    for (int it = 1; it <= maxit; it++) {
        const double xm = 0.5 * (a + b);
        const double tol1 = tol * fabs(x) + abst, tol2 = 2.0 * tol1;
        if (fabs(x - xm) <= (tol2 - 0.5 * (b - a))) {
            *xmin = x;
            *iters_out = it;
            return fx;
        }
        if (fabs(e) > tol1) {                           // try a parabolic step
            const double r = (x - w) * (fx - fv);
            double q = (x - v) * (fx - fw);
            double p = (x - v) * q - (x - w) * r;
            q = 2.0 * (q - r);
            if (q > 0.0) p = -p;
            q = fabs(q);
            const double etemp = e;
            e = d;
            if (fabs(p) >= fabs(0.5 * q * etemp) || p <= q * (a - x) || p >= q * (b - x)) {
                e = (x >= xm) ? a - x : b - x;          // golden-section step instead
                d = cgold * e;
            } else {
                d = p / q;
                const double u = x + d;
                if (u - a < tol2 || b - u < tol2) d = signed_mag(tol1, xm - x);
            }
        } else {
            e = (x >= xm) ? a - x : b - x;
            d = cgold * e;
        }
        const double u = (fabs(d) >= tol1) ? x + d : x + signed_mag(tol1, d);
        const double fu = f(u);
        if (fu <= fx) {
            if (u >= x) a = x; else b = x;
            v = w; w = x; x = u;
            fv = fw; fw = fx; fx = fu;
        } else {
            if (u < x) a = u; else b = u;
            if (fu <= fw || w == x) {
                v = w; w = u; fv = fw; fw = fu;
            } else if (fu <= fv || v == x || v == w) {
                v = u; fv = fu;
            }
        }
    }
    *xmin = x;
    *iters_out = -1;
    return fx;
}

struct CallbackObjective {
    shape_objective_fn fn;
    void *user;
    double operator()(double x) { return fn(x, user); }
};

}  // namespace
}  // namespace shape

using namespace shape;

extern "C" int shape_bracket_minimum(shape_objective_fn fn, void *user, double *ax, double *bx, double *cx,
                                     double *fa, double *fb, double *fc)
{
    if (!fn || !ax || !bx || !cx || !fa || !fb || !fc)
        return report_error(SHAPE_E_ARG, "shape_bracket_minimum: null argument");
    CallbackObjective f{fn, user};
    Bracket br{*ax, *bx, 0.0, 0.0, 0.0, 0.0};
    bracket_minimum(f, br);
    *ax = br.a; *bx = br.b; *cx = br.c; *fa = br.fa; *fb = br.fb; *fc = br.fc;
    return SHAPE_OK;
}

extern "C" int shape_brent_minimize(shape_objective_fn fn, void *user, double ax, double bx, double cx,
                                    double tol, double abstol, double *xmin, double *fmin)
{
    if (!fn || !xmin || !fmin) return report_error(SHAPE_E_ARG, "shape_brent_minimize: null argument");
    CallbackObjective f{fn, user};
    int iters;
    *fmin = brent_minimize(f, ax, bx, cx, tol, abstol, xmin, &iters);
    if (iters < 0) return report_error(SHAPE_E_TIMEOUT, "shape_brent_minimize: too many iterations");
    return iters;
}

namespace {

// Parameter access + objective of one fit. Engine-backed and callback-backed
// objectives share the iteration logic below.
struct FitTarget {
    virtual ~FitTarget() {}
    virtual int get(const shape_fit_param &p, int k, double *v) = 0;
    virtual int set(const shape_fit_param &p, int k, double v) = 0;
    // objective value; flags (posbnd, badradar) of the evaluation
    virtual int eval(double *obj, int *posbnd, int *badradar) = 0;
};

struct EngineTarget : FitTarget {
    shape_engine *e;
    int form;
    int get(const shape_fit_param &p, int, double *v) override
    {
        if (p.kind == SHAPE_PAR_SCALE) return shape_engine_get_scale(e, p.index, v);
        if (p.kind == SHAPE_PAR_VERTEX_R) return shape_engine_get_vertex_r(e, p.index, v);
        if (p.kind >= SHAPE_PAR_SPIN_ANGLE && p.kind <= SHAPE_PAR_OMEGAOFF)
            return shape_engine_get_spin_param(e, p.kind, p.index, v);
        return report_error(SHAPE_E_ARG, "bestfit: unknown parameter kind");
    }
    int set(const shape_fit_param &p, int, double v) override
    {
        if (p.kind == SHAPE_PAR_SCALE) return shape_engine_set_scale(e, p.index, v);
        if (p.kind == SHAPE_PAR_VERTEX_R) return shape_engine_set_vertex_r(e, p.index, v);
        if (p.kind >= SHAPE_PAR_SPIN_ANGLE && p.kind <= SHAPE_PAR_OMEGAOFF)
            return shape_engine_set_spin_param(e, p.kind, p.index, v);
        return report_error(SHAPE_E_ARG, "bestfit: unknown parameter kind");
    }
    // objective(x) of src/shape/bestfit.c:718-874 without penalties
    int eval(double *obj, int *posbnd, int *badradar) override
    {
        shape_eval_summary s;
        int rc = shape_engine_evaluate(e, form, &s);
        if (rc) return rc;
        *obj = s.objective;
        *posbnd = s.posbnd;
        *badradar = s.badradar;
        return SHAPE_OK;
    }
};

struct CallbackTarget : FitTarget {
    shape_param_objective_fn fn;
    void *user;
    double *values;
    int get(const shape_fit_param &, int k, double *v) override { *v = values[k]; return SHAPE_OK; }
    int set(const shape_fit_param &, int k, double v) override { values[k] = v; return SHAPE_OK; }
    int eval(double *obj, int *posbnd, int *badradar) override
    {
        *obj = fn(values, user, posbnd, badradar);
        return SHAPE_OK;
    }
};

// objective(x) for parameter k: set it, evaluate, record the trial
struct LineObjective {
    FitTarget &T;
    const shape_fit_param &P;
    int k;
    double *trace;
    int trace_max;
    int rc = SHAPE_OK, evaluations = 0, trace_n = 0, saw_posbnd = 0, saw_badradar = 0;
    double operator()(double x)
    {
        if (rc) return HUGE_VAL;
        if ((rc = T.set(P, k, x)) != SHAPE_OK) return HUGE_VAL;
        double obj;
        int pb = 0, br = 0;
        if ((rc = T.eval(&obj, &pb, &br)) != SHAPE_OK) return HUGE_VAL;
        evaluations++;
        saw_posbnd |= pb;
        saw_badradar |= br;
        if (trace && trace_n < trace_max) {
            trace[2 * trace_n] = k;
            trace[2 * trace_n + 1] = x;
            trace_n++;
        }
        return obj;
    }
};

// The iteration of bestfit (src/shape/bestfit.c:367-651) with first_fitpar
// = 0, no objfunc_start, no avoid_badpos and no term_badmodel: for each free
// parameter, bracket from (value, value + step), Brent-minimise, adopt the
// minimum; repeat while an iteration lowers the objective by at least
// term_prec (fractionally) and term_maxiter allows.
int fit_loop(FitTarget &T, const shape_fit_param *params, int nparams, const shape_fit_options *opt,
             shape_fit_result *res, double *trace, int trace_max)
{
    double enderr, beginerr;
    int pb, br;
    int rc = T.eval(&enderr, &pb, &br);
    if (rc) return rc;
    int iter = 0, evaluations = 1, trace_n = 0;
    res->initial_objective = enderr;
    bool keep;
    do {
        beginerr = enderr;
        iter++;
        for (int k = 0; k < nparams; k++) {
            const shape_fit_param &P = params[k];
            double cur;
            if ((rc = T.get(P, k, &cur)) != SHAPE_OK) return rc;
            LineObjective f{T, P, k, trace ? trace + 2 * trace_n : nullptr, trace ? trace_max - trace_n : 0};
            Bracket b{cur, cur + P.step, 0.0, 0.0, 0.0, 0.0};
            bracket_minimum(f, b);
            double xmin = cur;
            int iters = 0;
            if (!f.rc) enderr = brent_minimize(f, b.a, b.b, b.c, P.tol, P.abstol, &xmin, &iters);
            if (f.rc) return f.rc;
            if (iters < 0) return report_error(SHAPE_E_TIMEOUT, "bestfit: Brent minimisation did not converge");
            if ((rc = T.set(P, k, xmin)) != SHAPE_OK) return rc;
            evaluations += f.evaluations;
            trace_n += f.trace_n;
            // a model that left the POS window or the delay-Doppler frames in
            // some trial is evaluated once more at the adopted value
            // (src/shape/bestfit.c:581-582)
            if (f.saw_posbnd || f.saw_badradar) {
                double o;
                if ((rc = T.eval(&o, &pb, &br)) != SHAPE_OK) return rc;
                evaluations++;
            }
        }
        keep = (beginerr - enderr) / enderr >= opt->term_prec;
        if (opt->term_maxiter > 0 && iter >= opt->term_maxiter) keep = false;
    } while (keep);
    res->final_objective = enderr;
    res->iterations = iter;
    res->evaluations = evaluations;
    res->trace_len = trace_n;
    return SHAPE_OK;
}

}  // namespace

extern "C" int shape_engine_bestfit(shape_engine *e, const shape_fit_param *params, int nparams,
                                    const shape_fit_options *opt, shape_fit_result *res, double *trace,
                                    int trace_max)
{
    if (!e || !params || nparams <= 0 || !opt || !res)
        return report_error(SHAPE_E_ARG, "shape_engine_bestfit: invalid argument");
    EngineTarget T;
    T.e = e;
    T.form = opt->form;
    return fit_loop(T, params, nparams, opt, res, trace, trace_max);
}

extern "C" int shape_bestfit_host(shape_param_objective_fn fn, void *user, double *values,
                                  const shape_fit_param *params, int nparams, const shape_fit_options *opt,
                                  shape_fit_result *res, double *trace, int trace_max)
{
    if (!fn || !values || !params || nparams <= 0 || !opt || !res)
        return report_error(SHAPE_E_ARG, "shape_bestfit_host: invalid argument");
    CallbackTarget T;
    T.fn = fn;
    T.user = user;
    T.values = values;
    return fit_loop(T, params, nparams, opt, res, trace, trace_max);
}
