// SHAPE model files (.mod; read_mod, src/shape/read_mod.c:204-227) for the
// models the engine evaluates: one vertex component (read_shape, :289-542)
// with no component offsets, the homogeneous radar and optical scattering
// laws (read_photo, :544-1953) and the spin section (read_spin, :1954-2140),
// read and written; the data files of radar frames (delay-Doppler images
// and Doppler spectra, src/shape/read_dat.c:800-856, 1150-1176, 2074-2260);
// and the listfit output of a radar frame (.fitdat, src/shape/chi2.c:
// 525-560). Host code.
//
// The file is a stream of whitespace-separated tokens with comments in
// curly braces. A parameter is a state token (c, f or =) followed by its
// value. Numbers are converted with strtod / strtol and must be the whole
// token (src/util/getdouble.c, getint.c). Angles are stored in radians and
// spin rates in rad/day, by the same operations as read_spin, and the
// epochs in Julian days (cal2jd, src/astro/jdcal.c:8-13).
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "shape_b200.h"

namespace shape {
int report_error(int code, const std::string &msg);   // engine.cu
}

struct shape_mod_file {
    std::vector<double> a, u, r;
    // components back to back: vertices and facets of each, its scale
    // factors (3 each, with their states), linear offsets (km) and rotation
    // offsets (the file's degrees wrapped into (-180, 180], and in radians)
    std::vector<double> scale;
    std::vector<char> scale_state;
    std::vector<int> comp_nv, comp_nf;
    std::vector<double> comp_off, comp_rot, comp_rot_deg;
    std::vector<int> fv, af_ptr, af_idx;
    std::vector<char> r_state;
    std::vector<shape_radar_law> radar;
    std::vector<shape_optical_law> optical;
    std::vector<std::string> radar_state, optical_state;   // states of each law's parameters, in file order
    shape_spin_state spin;
    char angle_state[3], omega_state[3], inertia_state[3], omegadot_state[3], lib_state[3];
    char impulse_state[SHAPE_MAX_IMPULSES][3];
};

namespace {

const double D2R = 0.01745329251994330;   // src/shape/const.h

struct ParseError {
    int code;
    std::string msg;
};

class Tokens {
public:
    explicit Tokens(std::string text) : t_(std::move(text)) {}

    // The next token, or false at the end of the file.
    bool next(std::string &tok)
    {
        for (;;) {
            while (p_ < t_.size() && isspace((unsigned char)t_[p_])) {
                if (t_[p_] == '\n') line_++;
                p_++;
            }
            if (p_ < t_.size() && t_[p_] == '{') {
                while (p_ < t_.size() && t_[p_] != '}') {
                    if (t_[p_] == '\n') line_++;
                    p_++;
                }
                if (p_ >= t_.size()) fail("unclosed comment");
                p_++;
                continue;
            }
            break;
        }
        if (p_ >= t_.size()) return false;
        const size_t b = p_;
        while (p_ < t_.size() && !isspace((unsigned char)t_[p_]) && t_[p_] != '{') p_++;
        tok.assign(t_, b, p_ - b);
        return true;
    }
    std::string word(const char *what)
    {
        std::string s;
        if (!next(s)) fail(std::string("end of file instead of ") + what);
        return s;
    }
    int integer(const char *what)
    {
        const std::string s = word(what);
        char *end = nullptr;
        errno = 0;
        const long v = strtol(s.c_str(), &end, 10);
        if (*end != '\0' || errno == ERANGE || v < INT_MIN || v > INT_MAX)
            fail(std::string("expected an integer (") + what + "), got " + s);
        return (int)v;
    }
    double real(const char *what)
    {
        const std::string s = word(what);
        char *end = nullptr;
        const double v = strtod(s.c_str(), &end);
        if (*end != '\0') fail(std::string("expected a number (") + what + "), got " + s);
        return v;
    }
    // state (c, f or =) and value of a parameter
    double param(const char *what, char *state)
    {
        const std::string s = word(what);
        if (s != "c" && s != "f" && s != "=") fail(std::string("expected c, f or = before ") + what + ", got " + s);
        if (state) *state = s[0];
        return real(what);
    }
    [[noreturn]] void fail(const std::string &m, int code = SHAPE_E_ARG) const
    {
        throw ParseError{code, kind_ + " line " + std::to_string(line_) + ": " + m};
    }
    // the kind of file named in error messages
    void set_kind(const char *kind) { kind_ = kind; }

private:
    std::string t_;
    size_t p_ = 0;
    int line_ = 1;
    std::string kind_ = "model file";
};

// Julian day number of a calendar date at noon: Gregorian from 1582
// October 15 on, Julian before (Fliegel and Van Flandern 1968; the Julian
// calendar form of the same construction). Integer division truncates.
long julian_day_number(int yy, int mo, int dd)
{
    const bool gregorian = yy > 1582 || (yy == 1582 && (mo > 10 || (mo == 10 && dd >= 15)));
    const long y = yy, m = mo, d = dd;
    if (gregorian)
        return (1461 * (y + 4800 + (m - 14) / 12)) / 4 + (367 * (m - 2 - 12 * ((m - 14) / 12))) / 12 -
               (3 * ((y + 4900 + (m - 14) / 12) / 100)) / 4 + d - 32075;
    return 367 * y - (7 * (y + 5001 + (m - 9) / 7)) / 4 + (275 * m) / 9 + d + 1729777;
}

// Six integers yyyy mm dd hh mm ss -> Julian date (days).
double read_epoch(Tokens &tk, const char *what)
{
    int c[6];
    for (int i = 0; i < 6; i++) c[i] = tk.integer(what);
    if (c[0] <= 0 || c[1] < 1 || c[1] > 12 || c[2] < 1 || c[2] > 31) tk.fail(std::string("bad date in ") + what);
    double jd = (double)julian_day_number(c[0], c[1], c[2]) - 0.5;
    jd += ((c[3] * 60 + c[4]) * 60 + c[5]) / 86400.0;
    return jd;
}

// Julian date -> yyyy mm dd hh mm ss (Gregorian; the inverse of
// julian_day_number, Fliegel and Van Flandern 1968), seconds rounded as
// jd2cal rounds them (src/astro/jdcal.c:16-33). False before 1582 Oct 15.
bool calendar(double jd, int c[6])
{
    long jdn = (long)floor(jd + 0.5);
    long secs = (long)floor((jd + 0.5 - (double)jdn) * 86400 + 0.5);
    if (secs == 86400) { jdn++; secs = 0; }
    if (jdn < 2299161) return false;
    long l = jdn + 68569;
    const long n = 4 * l / 146097;
    l = l - (146097 * n + 3) / 4;
    const long i = 4000 * (l + 1) / 1461001;
    l = l - 1461 * i / 4 + 31;
    const long j = 80 * l / 2447;
    c[2] = (int)(l - 2447 * j / 80);
    l = j / 11;
    c[1] = (int)(j + 2 - 12 * l);
    c[0] = (int)(100 * (n - 49) + i + l);
    c[3] = (int)(secs / 3600);
    c[4] = (int)((secs % 3600) / 60);
    c[5] = (int)(secs % 60);
    return true;
}

void read_shape(Tokens &tk, shape_mod_file &m)
{
    const int ncomp = tk.integer("number of components");
    if (ncomp < 1) tk.fail("a model needs at least one component");
    for (int c = 0; c < ncomp; c++) {
        double off[3], deg[3];
        for (int j = 0; j < 6; j++) {
            char st;
            double v = tk.param(j < 3 ? "component offset" : "component rotation", &st);
            if (st != 'c')
                tk.fail("component offsets and rotations must be held constant (c)", SHAPE_E_UNSUPPORTED);
            // angles wrapped into (-180, 180] before the conversion
            // (src/shape/read_mod.c:314-320)
            if (j >= 3) v += 360.0 * floor((180.0 - v) / 360.0);
            if (j < 3) off[j] = v; else deg[j - 3] = v;
        }
        const std::string type = tk.word("component type");
        if (type != "vertex") tk.fail("component type " + type + ": only vertex components are supported",
                                      SHAPE_E_UNSUPPORTED);
        const int nv = tk.integer("number of vertices");
        if (nv < 4) tk.fail("a vertex model needs at least 4 vertices");
        const int v0 = (int)m.r.size(), f0 = (int)(m.fv.size() / 3);
        for (int j = 0; j < 3; j++) {
            char st;
            m.scale.push_back(tk.param("scale factor", &st));
            m.scale_state.push_back(st);
        }
        if (m.scale_state[3 * c] == '=') tk.fail("scale factor 0 cannot take the = state");
        m.a.resize(3 * (size_t)(v0 + nv));
        m.u.resize(3 * (size_t)(v0 + nv));
        m.r.resize(v0 + nv);
        m.r_state.resize(v0 + nv);
        for (int v = v0; v < v0 + nv; v++) {
            m.r[v] = tk.param("vertex deviation", &m.r_state[v]);
            if (m.r_state[v] == '=')
                tk.fail("mirrored vertex deviations (= state) are not supported", SHAPE_E_UNSUPPORTED);
            for (int k = 0; k < 3; k++) m.u[3 * (size_t)v + k] = tk.real("vertex direction");
            for (int k = 0; k < 3; k++) m.a[3 * (size_t)v + k] = tk.real("vertex base point");
        }
        const int nf = tk.integer("number of facets");
        if (nf < 4) tk.fail("a vertex model needs at least 4 facets");
        m.fv.resize(3 * (size_t)(f0 + nf));
        for (size_t k = 3 * (size_t)f0; k < m.fv.size(); k++) {
            const int v = tk.integer("facet vertex");
            if (v < 0 || v >= nv) tk.fail("facet vertex index out of range");
            m.fv[k] = v0 + v;                  // model-wide vertex index
        }
        m.comp_nv.push_back(nv);
        m.comp_nf.push_back(nf);
        for (int j = 0; j < 3; j++) {
            m.comp_off.push_back(off[j]);
            m.comp_rot_deg.push_back(deg[j]);
            m.comp_rot.push_back(deg[j] * D2R);
        }
    }
    // attached facets of each vertex, in increasing facet order
    // (setupvertices, src/shape/read_mod.c:2504-2590); a component's
    // vertices only touch its own facets
    const int nv = (int)m.r.size(), nf = (int)(m.fv.size() / 3);
    m.af_ptr.assign((size_t)nv + 1, 0);
    for (int v : m.fv) m.af_ptr[v + 1]++;
    for (int v = 0; v < nv; v++) m.af_ptr[v + 1] += m.af_ptr[v];
    m.af_idx.resize(m.fv.size());
    std::vector<int> fill(m.af_ptr.begin(), m.af_ptr.end() - 1);
    for (int f = 0; f < nf; f++)
        for (int k = 0; k < 3; k++) m.af_idx[fill[m.fv[3 * (size_t)f + k]]++] = f;
}

void read_photo(Tokens &tk, shape_mod_file &m)
{
    const int nrad = tk.integer("number of radar laws");
    if (nrad < 0) tk.fail("negative number of radar laws");
    for (int i = 0; i < nrad; i++) {
        const std::string s = tk.word("radar law");
        shape_radar_law L;
        memset(&L, 0, sizeof L);
        std::string states;
        auto par = [&](const char *what) {
            char st;
            const double v = tk.param(what, &st);
            states.push_back(st);
            return v;
        };
        auto cutoff = [&]() {
            const double deg = tk.real("cutoff angle");
            if (deg <= 0.0 || deg > 90.0) tk.fail("cutoff angle must be in (0, 90] deg");
            return cos(deg * D2R);
        };
        if (s == "none") {
            L.type = 0;
        } else if (s == "cosine") {
            L.type = SHAPE_RADLAW_COSINE_DIFF;
            L.diff_R = par("R");
            L.diff_C = par("C");
        } else if (s == "gaussian" || s == "hagfors" || s == "cosine_qs") {
            L.type = s == "gaussian" ? SHAPE_RADLAW_GAUSSIAN : s == "hagfors" ? SHAPE_RADLAW_HAGFORS
                                                                               : SHAPE_RADLAW_COSINE_QS;
            L.qs_R = par("R");
            L.qs_C = par("C");
            L.qs_cos_cutoff = cutoff();
        } else if (s == "gauss+cosine" || s == "hagfors+cosine" || s == "cosine+cosine") {
            L.type = s == "gauss+cosine" ? SHAPE_RADLAW_GAUSSIAN_COSINE
                     : s == "hagfors+cosine" ? SHAPE_RADLAW_HAGFORS_COSINE : SHAPE_RADLAW_COSINE_COSINE;
            L.qs_R = par("R");
            L.qs_C = par("C");
            L.qs_cos_cutoff = cutoff();
            L.diff_R = par("R");
            L.diff_C = par("C");
        } else {
            tk.fail("radar law " + s + " is not supported", SHAPE_E_UNSUPPORTED);
        }
        m.radar.push_back(L);
        m.radar_state.push_back(states);
    }
    const int nopt = tk.integer("number of optical laws");
    if (nopt < 0) tk.fail("negative number of optical laws");
    for (int i = 0; i < nopt; i++) {
        const std::string s = tk.word("optical law");
        shape_optical_law L;
        memset(&L, 0, sizeof L);
        std::string states;
        auto par = [&](const char *what) {
            char st;
            const double v = tk.param(what, &st);
            states.push_back(st);
            return v;
        };
        if (s == "none") {
            L.type = 0;
        } else if (s == "lambertian" || s == "lommel") {
            L.type = s == "lambertian" ? SHAPE_OPTLAW_LAMBERT : SHAPE_OPTLAW_LOMMEL;
            L.R = par("R");
        } else if (s == "kaasalainen") {
            L.type = SHAPE_OPTLAW_KAASALAINEN;
            L.R = par("R");
            L.wt = par("wt");
            L.A0 = par("A0");
            L.D = par("D");
            L.k = par("k");
            L.D *= D2R;
            L.k /= D2R;
        } else {
            tk.fail("optical law " + s + " is not supported", SHAPE_E_UNSUPPORTED);
        }
        m.optical.push_back(L);
        m.optical_state.push_back(states);
    }
}

void read_spin(Tokens &tk, shape_mod_file &m)
{
    shape_spin_state &sp = m.spin;
    memset(&sp, 0, sizeof sp);
    sp.t0 = read_epoch(tk, "spin epoch");
    for (int i = 0; i < 3; i++) sp.angle[i] = tk.param("spin angle", &m.angle_state[i]);
    for (int i = 0; i < 3; i++) sp.omega[i] = tk.param("spin rate", &m.omega_state[i]);
    for (int i = 0; i < 3; i++) sp.inertia[i] = tk.param("moment of inertia", &m.inertia_state[i]);
    for (int i = 0; i < 3; i++) sp.omegadot[i] = tk.param("spin-rate change", &m.omegadot_state[i]);
    sp.lib_amp = tk.param("libration amplitude", &m.lib_state[0]);
    sp.lib_freq = tk.param("libration frequency", &m.lib_state[1]);
    sp.lib_phase = tk.param("libration phase", &m.lib_state[2]);
    sp.n_impulse = tk.integer("number of spin impulses");
    if (sp.n_impulse < 0 || sp.n_impulse > SHAPE_MAX_IMPULSES) tk.fail("too many spin impulses");
    for (int n = 0; n < sp.n_impulse; n++) {
        sp.t_impulse[n] = read_epoch(tk, "spin impulse epoch");
        if (n > 0 && sp.t_impulse[n] <= sp.t_impulse[n - 1])
            tk.fail("spin impulses must be in increasing chronological order");
        for (int i = 0; i < 3; i++) sp.impulse[n][i] = tk.param("spin impulse", &m.impulse_state[n][i]);
    }
    // principal-axis rotator: x and y spin held at zero and no x/y impulses
    // (src/shape/read_mod.c:2060-2080)
    sp.pa = 0;
    if (sp.omega[0] == 0.0 && m.omega_state[0] == 'c' && sp.omega[1] == 0.0 && m.omega_state[1] == 'c') {
        sp.pa = 1;
        for (int n = 0; n < sp.n_impulse && sp.pa; n++)
            if (sp.impulse[n][0] != 0.0 || m.impulse_state[n][0] == 'f' || sp.impulse[n][1] != 0.0 ||
                m.impulse_state[n][1] == 'f')
                sp.pa = 0;
    }
    const bool xy_dot = sp.omegadot[0] != 0 || m.omegadot_state[0] == 'f' || sp.omegadot[1] != 0 ||
                        m.omegadot_state[1] == 'f';
    if (sp.pa && xy_dot) tk.fail("a principal-axis rotator cannot have x or y spin-rate change");
    if (!sp.pa && (xy_dot || sp.omegadot[2] != 0 || m.omegadot_state[2] == 'f' || sp.lib_amp != 0 ||
                   m.lib_state[0] == 'f'))
        tk.fail("a non-principal-axis rotator cannot have spin-rate change or libration");
    // Euler angles "over the pole" folded back, all angles into [0, 360)
    // deg, then radians and rad/day (src/shape/read_mod.c:2113-2135)
    sp.angle[1] -= 360.0 * floor(sp.angle[1] / 360.0);
    if (sp.angle[1] > 180.0) {
        sp.angle[1] = 360.0 - sp.angle[1];
        sp.angle[0] += 180.0;
        sp.angle[2] += 180.0;
    }
    for (int i = 0; i < 3; i++) {
        sp.angle[i] -= 360.0 * floor(sp.angle[i] / 360.0);
        sp.angle[i] *= D2R;
        sp.omega[i] *= D2R;
        sp.omegadot[i] *= D2R;
        for (int n = 0; n < sp.n_impulse; n++) sp.impulse[n][i] *= D2R;
    }
    sp.lib_amp *= D2R;
    sp.lib_freq *= D2R;
    sp.lib_phase *= D2R;
}

}  // namespace

extern "C" {

int shape_mod_read(const char *path, shape_mod_file **out)
{
    if (!path || !out) return shape::report_error(SHAPE_E_ARG, "mod_read: null argument");
    *out = nullptr;
    FILE *fp = fopen(path, "rb");
    if (!fp) return shape::report_error(SHAPE_E_ARG, std::string("mod_read: cannot open ") + path);
    std::string text;
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, n);
    fclose(fp);
    shape_mod_file *m = new shape_mod_file();
    memset(m->impulse_state, 'c', sizeof m->impulse_state);
    try {
        Tokens tk(std::move(text));
        read_shape(tk, *m);
        read_photo(tk, *m);
        read_spin(tk, *m);
    } catch (const ParseError &e) {
        delete m;
        return shape::report_error(e.code, e.msg);
    }
    *out = m;
    return SHAPE_OK;
}

void shape_mod_free(shape_mod_file *m) { delete m; }

int shape_mod_model(const shape_mod_file *m, shape_model_desc *out)
{
    if (!m || !out) return shape::report_error(SHAPE_E_ARG, "mod_model: null argument");
    out->nv = (int)m->r.size();
    out->nf = (int)(m->fv.size() / 3);
    out->a = m->a.data();
    out->u = m->u.data();
    out->r = m->r.data();
    for (int j = 0; j < 3; j++) out->scale[j] = m->scale[j];
    out->fv = m->fv.data();
    out->af_ptr = m->af_ptr.data();
    out->af_idx = m->af_idx.data();
    const int nc = (int)m->comp_nv.size();
    out->ncomp = nc > 1 ? nc : 0;
    out->comp_nv = nc > 1 ? m->comp_nv.data() : nullptr;
    out->comp_nf = nc > 1 ? m->comp_nf.data() : nullptr;
    out->comp_scale = nc > 1 ? m->scale.data() : nullptr;
    out->comp_rot = nc > 1 ? m->comp_rot.data() : nullptr;
    out->comp_off = nc > 1 ? m->comp_off.data() : nullptr;
    return SHAPE_OK;
}

int shape_mod_radar_law(const shape_mod_file *m, int ilaw, shape_radar_law *law)
{
    if (!m) return shape::report_error(SHAPE_E_ARG, "mod_radar_law: null argument");
    if (!law) return (int)m->radar.size();
    if (ilaw < 0 || ilaw >= (int)m->radar.size()) return shape::report_error(SHAPE_E_ARG, "mod_radar_law: no such law");
    *law = m->radar[ilaw];
    return (int)m->radar.size();
}

int shape_mod_optical_law(const shape_mod_file *m, int ilaw, shape_optical_law *law)
{
    if (!m) return shape::report_error(SHAPE_E_ARG, "mod_optical_law: null argument");
    if (!law) return (int)m->optical.size();
    if (ilaw < 0 || ilaw >= (int)m->optical.size())
        return shape::report_error(SHAPE_E_ARG, "mod_optical_law: no such law");
    *law = m->optical[ilaw];
    return (int)m->optical.size();
}

int shape_mod_spin(const shape_mod_file *m, shape_spin_state *spin)
{
    if (!m || !spin) return shape::report_error(SHAPE_E_ARG, "mod_spin: null argument");
    *spin = m->spin;
    return SHAPE_OK;
}

int shape_mod_free_params(const shape_mod_file *m, shape_fit_param *out, int max)
{
    if (!m || (max > 0 && !out)) return shape::report_error(SHAPE_E_ARG, "mod_free_params: null argument");
    int n = 0;
    auto add = [&](char state, int kind, int index) {
        if (state != 'f') return;
        if (n < max) {
            out[n].kind = kind;
            out[n].index = index;
            out[n].step = out[n].tol = out[n].abstol = 0.0;
        }
        n++;
    };
    // per component its scale factors, then its vertex deviations
    // (src/shape/mkparlist.c:109-235)
    for (size_t c = 0, v0 = 0; c < m->comp_nv.size(); v0 += m->comp_nv[c], c++) {
        for (int j = 0; j < 3; j++) add(m->scale_state[3 * c + j], SHAPE_PAR_SCALE, (int)(3 * c + j));
        for (size_t v = v0; v < v0 + m->comp_nv[c]; v++) add(m->r_state[v], SHAPE_PAR_VERTEX_R, (int)v);
    }
    for (int i = 0; i < 3; i++) add(m->angle_state[i], SHAPE_PAR_SPIN_ANGLE, i);
    for (int i = 0; i < 3; i++) add(m->omega_state[i], SHAPE_PAR_SPIN_OMEGA, i);
    for (int i = 0; i < 3; i++) add(m->inertia_state[i], SHAPE_PAR_SPIN_INERTIA, i);
    for (int i = 0; i < 3; i++) add(m->omegadot_state[i], SHAPE_PAR_SPIN_OMEGADOT, i);
    for (int k = 0; k < m->spin.n_impulse; k++)
        for (int i = 0; i < 3; i++) add(m->impulse_state[k][i], SHAPE_PAR_SPIN_IMPULSE, 3 * k + i);
    for (int i = 0; i < 3; i++) add(m->lib_state[i], SHAPE_PAR_SPIN_LIB, i);
    return n;
}

// Writes m as a model file that read_mod reads back: its vertex components
// with their offsets, its laws and the spin section, the parameter states of
// the file it came from, numbers with 17 significant digits (shape values
// exactly; angles and rates back in degrees, which rounds their last bit).
int shape_mod_write(const shape_mod_file *m, const char *path)
{
    if (!m || !path) return shape::report_error(SHAPE_E_ARG, "mod_write: null argument");
    int t0[6], ti[SHAPE_MAX_IMPULSES][6];
    const shape_spin_state &sp = m->spin;
    bool ok = calendar(sp.t0, t0);
    for (int n = 0; n < sp.n_impulse; n++) ok = ok && calendar(sp.t_impulse[n], ti[n]);
    if (!ok) return shape::report_error(SHAPE_E_UNSUPPORTED, "mod_write: epoch before the Gregorian calendar");
    FILE *fp = fopen(path, "w");
    if (!fp) return shape::report_error(SHAPE_E_ARG, std::string("mod_write: cannot create ") + path);
    auto par = [&](char st, double v) { fprintf(fp, " %c %.17g", st, v); };
    const int ncomp = (int)m->comp_nv.size();
    fprintf(fp, "{SHAPE model file written by shape-b200}\n\n{shape}\n%d {components}\n", ncomp);
    int v0 = 0, f0 = 0;
    for (int c = 0; c < ncomp; c++) {
        const int nv = m->comp_nv[c], nf = m->comp_nf[c];
        for (int j = 0; j < 3; j++) par('c', m->comp_off[3 * (size_t)c + j]);
        fprintf(fp, " {linear offsets (km)}\n");
        for (int j = 0; j < 3; j++) par('c', m->comp_rot_deg[3 * (size_t)c + j]);
        fprintf(fp, " {rotation offsets (deg)}\n");
        fprintf(fp, "vertex\n%d {vertices}\n", nv);
        for (int j = 0; j < 3; j++) par(m->scale_state[3 * (size_t)c + j], m->scale[3 * (size_t)c + j]);
        fprintf(fp, " {scale factors}\n");
        for (int v = v0; v < v0 + nv; v++) {
            par(m->r_state[v], m->r[v]);
            for (int k = 0; k < 3; k++) fprintf(fp, " %.17g", m->u[3 * (size_t)v + k]);
            for (int k = 0; k < 3; k++) fprintf(fp, " %.17g", m->a[3 * (size_t)v + k]);
            fprintf(fp, "\n");
        }
        fprintf(fp, "%d {facets}\n", nf);
        for (int f = f0; f < f0 + nf; f++)
            fprintf(fp, "%d %d %d\n", m->fv[3 * (size_t)f] - v0, m->fv[3 * (size_t)f + 1] - v0,
                    m->fv[3 * (size_t)f + 2] - v0);
        v0 += nv;
        f0 += nf;
    }
    fprintf(fp, "\n{photometry}\n%d {radar laws}\n", (int)m->radar.size());
    for (size_t i = 0; i < m->radar.size(); i++) {
        const shape_radar_law &L = m->radar[i];
        const std::string &st = m->radar_state[i];
        const double cut = acos(L.qs_cos_cutoff) / D2R;
        switch (L.type) {
        case SHAPE_RADLAW_COSINE_DIFF:
            fprintf(fp, "cosine"); par(st[0], L.diff_R); par(st[1], L.diff_C); break;
        case SHAPE_RADLAW_GAUSSIAN: case SHAPE_RADLAW_HAGFORS: case SHAPE_RADLAW_COSINE_QS:
            fprintf(fp, L.type == SHAPE_RADLAW_GAUSSIAN ? "gaussian" : L.type == SHAPE_RADLAW_HAGFORS ? "hagfors"
                                                                                                       : "cosine_qs");
            par(st[0], L.qs_R); par(st[1], L.qs_C); fprintf(fp, " %.17g", cut); break;
        case SHAPE_RADLAW_GAUSSIAN_COSINE: case SHAPE_RADLAW_HAGFORS_COSINE: case SHAPE_RADLAW_COSINE_COSINE:
            fprintf(fp, L.type == SHAPE_RADLAW_GAUSSIAN_COSINE ? "gauss+cosine"
                        : L.type == SHAPE_RADLAW_HAGFORS_COSINE ? "hagfors+cosine" : "cosine+cosine");
            par(st[0], L.qs_R); par(st[1], L.qs_C); fprintf(fp, " %.17g", cut);
            par(st[2], L.diff_R); par(st[3], L.diff_C); break;
        default:
            fprintf(fp, "none");
        }
        fprintf(fp, "\n");
    }
    fprintf(fp, "%d {optical laws}\n", (int)m->optical.size());
    for (size_t i = 0; i < m->optical.size(); i++) {
        const shape_optical_law &L = m->optical[i];
        const std::string &st = m->optical_state[i];
        if (L.type == SHAPE_OPTLAW_LAMBERT || L.type == SHAPE_OPTLAW_LOMMEL) {
            fprintf(fp, L.type == SHAPE_OPTLAW_LAMBERT ? "lambertian" : "lommel");
            par(st[0], L.R);
        } else if (L.type == SHAPE_OPTLAW_KAASALAINEN) {
            fprintf(fp, "kaasalainen");
            par(st[0], L.R); par(st[1], L.wt); par(st[2], L.A0); par(st[3], L.D / D2R); par(st[4], L.k * D2R);
        } else {
            fprintf(fp, "none");
        }
        fprintf(fp, "\n");
    }
    fprintf(fp, "\n{spin}\n%d %d %d %d %d %d {t0}\n", t0[0], t0[1], t0[2], t0[3], t0[4], t0[5]);
    for (int i = 0; i < 3; i++) par(m->angle_state[i], sp.angle[i] / D2R);
    fprintf(fp, " {angles (deg)}\n");
    for (int i = 0; i < 3; i++) par(m->omega_state[i], sp.omega[i] / D2R);
    fprintf(fp, " {spin (deg/day)}\n");
    for (int i = 0; i < 3; i++) par(m->inertia_state[i], sp.inertia[i]);
    fprintf(fp, " {moments of inertia}\n");
    for (int i = 0; i < 3; i++) par(m->omegadot_state[i], sp.omegadot[i] / D2R);
    fprintf(fp, " {spin change (deg/day/day)}\n");
    par(m->lib_state[0], sp.lib_amp / D2R);
    par(m->lib_state[1], sp.lib_freq / D2R);
    par(m->lib_state[2], sp.lib_phase / D2R);
    fprintf(fp, " {libration}\n%d {spin impulses}\n", sp.n_impulse);
    for (int n = 0; n < sp.n_impulse; n++) {
        fprintf(fp, "%d %d %d %d %d %d", ti[n][0], ti[n][1], ti[n][2], ti[n][3], ti[n][4], ti[n][5]);
        for (int i = 0; i < 3; i++) par(m->impulse_state[n][i], sp.impulse[n][i] / D2R);
        fprintf(fp, "\n");
    }
    const int bad = ferror(fp);
    if (fclose(fp) != 0 || bad) return shape::report_error(SHAPE_E_ARG, std::string("mod_write: write failed: ") + path);
    return SHAPE_OK;
}

// The engine's current scale factors, vertex deviations and (with a spin
// model) spin parameters into m, as a fit leaves them.
int shape_mod_take_engine(shape_mod_file *m, shape_engine *e)
{
    if (!m || !e) return shape::report_error(SHAPE_E_ARG, "mod_take_engine: null argument");
    for (size_t j = 0; j < m->scale.size(); j++)
        if (int rc = shape_engine_get_scale(e, (int)j, &m->scale[j])) return rc;
    for (size_t v = 0; v < m->r.size(); v++)
        if (int rc = shape_engine_get_vertex_r(e, (int)v, &m->r[v])) return rc;
    double x;
    if (shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_ANGLE, 0, &x) != SHAPE_OK) return SHAPE_OK;   // no spin model
    shape_spin_state &sp = m->spin;
    for (int i = 0; i < 3; i++) {
        shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_ANGLE, i, &sp.angle[i]);
        shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_OMEGA, i, &sp.omega[i]);
        shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_INERTIA, i, &sp.inertia[i]);
        shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_OMEGADOT, i, &sp.omegadot[i]);
    }
    for (int k = 0; k < 3 * sp.n_impulse; k++)
        shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_IMPULSE, k, &sp.impulse[k / 3][k % 3]);
    shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_LIB, 0, &sp.lib_amp);
    shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_LIB, 1, &sp.lib_freq);
    shape_engine_get_spin_param(e, SHAPE_PAR_SPIN_LIB, 2, &sp.lib_phase);
    return SHAPE_OK;
}

// One radar data file (a delay-Doppler image of ndel x ndop, or a Doppler
// spectrum as ndel = 1), as read_deldop / read_doppler read it
// (src/shape/read_dat.c:800-856, 1150-1176): the type from the first 128
// bytes (any byte >= 128: raw float32; "SIMPLE": FITS, not supported;
// "type" in any case: an RDF header, lines up to one that starts with '.',
// then float32; otherwise ASCII numbers with comments in curly braces),
// each value rounded to float, the window idel_use x idop_use (1-based,
// inclusive) kept and multiplied by sdev; then per kept pixel the gamma
// transform (value > 0: value^(1/gamma); delay-Doppler data only) and
// 1/variance = 1/sdev^2, or 1/(sdev^2 + (obs/sqrt(nlooks))^2) with speckle
// (nlooks > 0), times pixweight of the pixel (full-size array, or null).
int shape_read_radar_data(const char *path, int ndel, int ndop, const int idel_use[2], const int idop_use[2],
                          int big_endian, double sdev, double gamma, double nlooks, const double *pixweight,
                          double *obs, double *oneovervar)
{
    if (!path || !idel_use || !idop_use || !obs || !oneovervar || ndel < 1 || ndop < 1 ||
        idel_use[0] < 1 || idel_use[1] > ndel || idel_use[0] > idel_use[1] || idop_use[0] < 1 ||
        idop_use[1] > ndop || idop_use[0] > idop_use[1] || !(gamma > 0.0))
        return shape::report_error(SHAPE_E_ARG, "read_radar_data: invalid argument");
    FILE *fp = fopen(path, "rb");
    if (!fp) return shape::report_error(SHAPE_E_ARG, std::string("read_radar_data: cannot open ") + path);
    std::string text;
    char buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, n);
    fclose(fp);
    if (text.size() < 128) return shape::report_error(SHAPE_E_ARG, "read_radar_data: file shorter than 128 bytes");
    bool binary = false;
    for (int j = 0; j < 128; j++) binary = binary || (unsigned char)text[j] >= 128;
    std::string head(text.data(), strnlen(text.data(), 128));
    const bool fits = !binary && head.find("SIMPLE") != std::string::npos;
    for (char &c : head) c = (char)tolower((unsigned char)c);
    const bool rdf = !binary && !fits && head.find("type") != std::string::npos;
    if (fits) return shape::report_error(SHAPE_E_UNSUPPORTED, "read_radar_data: FITS data files are not supported");
    const int wdop = idop_use[1] - idop_use[0] + 1;
    const size_t total = (size_t)ndel * ndop;
    std::vector<float> px(total);
    if (binary || rdf) {
        size_t off = 0;
        if (rdf) {                                   // header lines, read as fgets reads them (199 bytes at most)
            for (;;) {
                if (off >= text.size()) return shape::report_error(SHAPE_E_ARG, "read_radar_data: RDF header without end");
                const size_t nl = text.find('\n', off);
                const size_t end = std::min(nl == std::string::npos ? text.size() : nl + 1, off + 199);
                const char first = text[off];
                off = end;
                if (first == '.') break;
            }
        }
        if (text.size() - off < total * sizeof(float))
            return shape::report_error(SHAPE_E_ARG, "read_radar_data: data file too short");
        memcpy(px.data(), text.data() + off, total * sizeof(float));
        const uint16_t one = 1;
        const bool little_host = *(const unsigned char *)&one == 1;
        if (little_host == (big_endian != 0))
            for (float &v : px) {
                unsigned char *b = (unsigned char *)&v;
                std::swap(b[0], b[3]);
                std::swap(b[1], b[2]);
            }
    } else {
        try {
            Tokens tk(std::move(text));
            for (size_t k = 0; k < total; k++) px[k] = (float)tk.real("data value");
        } catch (const ParseError &e) {
            return shape::report_error(e.code, "read_radar_data: " + e.msg);
        }
    }
    const double lookfact = nlooks > 0.0 ? 1 / sqrt(nlooks) : 0.0;
    for (int j = idel_use[0]; j <= idel_use[1]; j++)
        for (int k = idop_use[0]; k <= idop_use[1]; k++) {
            const size_t src = (size_t)(j - 1) * ndop + (k - 1);
            const size_t dst = (size_t)(j - idel_use[0]) * wdop + (k - idop_use[0]);
            double o = px[src] * sdev;
            if (gamma != 1.0 && o > 0.0) o = pow(o, 1 / gamma);
            obs[dst] = o;
            double w = nlooks > 0.0 ? 1 / (pow(sdev, 2.0) + pow(lookfact * o, 2.0)) : 1 / pow(sdev, 2.0);
            if (pixweight) w *= pixweight[src];
            oneovervar[dst] = w;
        }
    return SHAPE_OK;
}

// A lightcurve data file (read_lghtcrv, src/shape/read_dat.c:1925-1956): n
// points of (epoch JD, magnitude, magnitude error) as tokens; intensity
// relative to the Sun exp(-0.4 ln10 (mag - sun_appmag)), its error
// 0.4 ln10 magerr intensity, and 1/variance.
int shape_read_lghtcrv_data(const char *path, int n, double sun_appmag, double *t, double *obs,
                            double *oneovervar)
{
    if (!path || n < 1 || !t || !obs || !oneovervar)
        return shape::report_error(SHAPE_E_ARG, "read_lghtcrv_data: invalid argument");
    FILE *fp = fopen(path, "rb");
    if (!fp) return shape::report_error(SHAPE_E_ARG, std::string("read_lghtcrv_data: cannot open ") + path);
    std::string text;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, got);
    fclose(fp);
    const double LN10 = 2.302585092994046;   // src/shape/const.h
    try {
        Tokens tk(std::move(text));
        for (int i = 0; i < n; i++) {
            const double epoch = tk.real("epoch");
            const double mag = tk.real("magnitude");
            const double magerr = tk.real("magnitude error");
            const double intens = exp(-0.4 * LN10 * (mag - sun_appmag));
            const double err = (0.4 * LN10 * magerr) * intens;
            t[i] = epoch;
            obs[i] = intens;
            oneovervar[i] = 1.0 / (err * err);
        }
    } catch (const ParseError &e) {
        return shape::report_error(e.code, "read_lghtcrv_data: " + e.msg);
    }
    return SHAPE_OK;
}

}  // extern "C"

// ------------------------------------------------------------- .obs files

struct shape_obs_file {
    struct Frame {
        std::string name;
        double t0, sdev, cal, nlooks, delcom, weight;
        char cal_state;
        // pixel-weighting mask (src/shape/read_dat.c:696-762, 1059-1118):
        // its weights (delay-major, the full image), or empty when the
        // frame has none or its mask file is not loaded; the window of
        // positive weights (1-based, inclusive: delay, then Doppler) and
        // the frame's dof
        int weighted = 0;
        std::vector<double> mask;
        int win[4] = {1, 1, 1, 1};
        double dof = 0.0;
    };
    struct Set {
        int doppler = 0;                 // 1: a Doppler set (read_doppler)
        int lightcurve = 0;              // 1: a lightcurve or heliocurve set (read_lghtcrv)
        int iradlaw;
        double angleoff[3], omegaoff[3];
        char angle_state[3], omega_state[3];   // c, f or = (= ties to an earlier set)
        char delcor_state;                     // state of the first delay-correction coefficient
        std::vector<shape_ephem_point> ephem;
        shape_deldop_set dd;
        int ndel, ndop;
        double dopcom, dopDC;
        double delcor_t0;
        std::vector<double> delcor;
        std::string dir;
        std::vector<Frame> frames;
        // smearing (src/shape/read_dat.c:635-646): views per frame, the
        // epoch view's index and the interval between views in days
        int nviews = 1, v0 = 0;
        double view_interval = 0.0;
        // lightcurve sets (read_lghtcrv, src/shape/read_dat.c:1667-2063)
        int ioptlaw = 0;
        std::vector<shape_ephem_point> solephem;   // the Sun as seen by the observer
        std::vector<double> x0;                    // calculated epochs before light-time correction
        std::string lcname;                        // data file
        char lc_cal_state = 'c';
        double lc_cal = 0.0, lc_weight = 0.0;
        std::vector<double> lc_t0, lc_mag, lc_magerr;   // the data file's points
        // plane-of-sky sets (read_poset, src/shape/read_dat.c:1392-1560)
        int poset = 0;
        double angle_per_pixel = 0.0;    // radians
        struct PosFrame {
            std::string name;            // image file (FITS) in dir
            double t0, northangle, off[2], weight;
            int pixels_weighted;
        };
        std::vector<PosFrame> pframes;
    };
    std::vector<Set> sets;
    std::string maskdir;                 // "" : the sets' data directories
};

// An ephemeris table: a count, then per entry an epoch (yyyy mm dd hh mm
// ss), RA and Dec in degrees and distance in AU.
static std::vector<shape_ephem_point> read_ephem(Tokens &tk, const char *what)
{
    const int ne = tk.integer(what);
    if (ne < 2) tk.fail(std::string(what) + ": an ephemeris needs at least 2 points");
    std::vector<shape_ephem_point> v(ne);
    for (int i = 0; i < ne; i++) {
        v[i].t = read_epoch(tk, "ephemeris epoch");
        v[i].ra = tk.real("RA") * D2R;
        v[i].dec = tk.real("Dec") * D2R;
        v[i].dist = tk.real("distance");
    }
    return v;
}

// The body of a plane-of-sky set (read_poset,
// src/shape/read_dat.c:1392-1460): optical law, the asteroid's and the
// Sun's ephemerides, the angular pixel size (arcsec), the smearing line,
// the data directory and per frame its image file, epoch, north angle
// (degrees), COM offsets (fit-grid pixels, free parameters), weight and
// pixel-weighting flag. The images are FITS files, which this reader does
// not open.
static void read_poset_set(Tokens &tk, shape_obs_file::Set &S)
{
    S.poset = 1;
    S.delcor_state = 'c';
    memset(&S.dd, 0, sizeof S.dd);
    S.ndel = S.ndop = 0;
    S.iradlaw = 0;
    S.ioptlaw = tk.integer("optical law");
    if (S.ioptlaw < 0) tk.fail("negative optical law index");
    S.ephem = read_ephem(tk, "asteroid ephemeris points");
    S.solephem = read_ephem(tk, "solar ephemeris points");
    S.angle_per_pixel = (tk.real("angular pixel size") / 3600) * D2R;
    S.nviews = tk.integer("views per frame");
    if (S.nviews < 1) tk.fail("views per frame must be at least 1");
    S.view_interval = tk.real("view interval") / 86400;
    const std::string mode = tk.word("smearing mode");
    if (mode == "center") S.v0 = S.nviews / 2;
    else if (mode == "first") S.v0 = 0;
    else tk.fail("smearing mode " + mode + " is not supported", SHAPE_E_UNSUPPORTED);
    S.dir = tk.word("data directory");
    const int nfr = tk.integer("frames");
    if (nfr < 1) tk.fail("a set needs at least one frame");
    for (int i = 0; i < nfr; i++) {
        shape_obs_file::Set::PosFrame F;
        F.name = tk.word("image file");
        F.t0 = read_epoch(tk, "frame epoch");
        F.northangle = tk.real("north angle") * D2R;
        char st;
        F.off[0] = tk.param("x offset", &st);
        F.off[1] = tk.param("y offset", &st);
        F.weight = tk.real("frame weight");
        F.pixels_weighted = tk.integer("pixel-weighting flag");
        S.pframes.push_back(F);
    }
}

// The body of a lightcurve or heliocurve set (read_lghtcrv,
// src/shape/read_dat.c:1667-1956): optical law, the asteroid's and the
// Sun's ephemerides, the calculated epochs (a list, a start / stop / step,
// or the observation epochs), one view per point, the data file and its
// calibration and weight; the data file is read here, as read_dat reads
// it, so a set whose calculated epochs are its observation epochs knows
// them. A heliocurve set is read exactly as a lightcurve set: read_dat
// gives read_lghtcrv the set type LGHTCRV for both (:487-502), so the
// reference never takes read_lghtcrv's heliocentric branch (:1740-1786)
// and uses the two tables as written.
static void read_lghtcrv_set(Tokens &tk, shape_obs_file::Set &S)
{
    S.lightcurve = 1;
    S.delcor_state = 'c';
    memset(&S.dd, 0, sizeof S.dd);
    S.ndel = S.ndop = 0;
    S.iradlaw = 0;
    S.ioptlaw = tk.integer("optical law");
    if (S.ioptlaw < 0) tk.fail("negative optical law index");
    S.ephem = read_ephem(tk, "asteroid ephemeris points");
    S.solephem = read_ephem(tk, "solar ephemeris points");
    const int np = tk.integer("calculation epochs");
    if (np > 0) {
        for (int i = 0; i < np; i++) {
            S.x0.push_back(tk.real("calculation epoch"));
            if (i > 0 && S.x0[i] <= S.x0[i - 1]) tk.fail("calculation epochs must increase");
        }
    } else if (np == 0) {
        const double t1 = tk.real("start epoch"), t2 = tk.real("stop epoch"), dt = tk.real("epoch step");
        if (t2 < t1 || dt <= 0) tk.fail("calculation epochs: need stop >= start and step > 0");
        const int nc = ((int)floor((t2 - t1) / dt)) + 1;
        for (int i = 1; i <= nc; i++) S.x0.push_back(t1 + (i - 1) * dt);
    }
    const int nviews = tk.integer("views per point");
    tk.real("view interval");
    const std::string smear = tk.word("smearing mode");
    if (smear != "center" && smear != "first") tk.fail("smearing mode " + smear + " is not known");
    if (nviews != 1) tk.fail("smeared points (more than one view) are not supported", SHAPE_E_UNSUPPORTED);
    const int n = tk.integer("lightcurve points");
    if (n < 1) tk.fail("a lightcurve needs at least one point");
    S.lcname = tk.word("lightcurve data file");
    S.lc_cal = tk.param("calibration", &S.lc_cal_state);
    S.lc_weight = tk.real("weight");
    FILE *fp = fopen(S.lcname.c_str(), "rb");
    if (!fp) tk.fail("cannot open lightcurve data file " + S.lcname);
    std::string text;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, got);
    fclose(fp);
    Tokens dt(std::move(text));
    dt.set_kind("lightcurve data file");
    for (int i = 0; i < n; i++) {
        S.lc_t0.push_back(dt.real("epoch"));
        S.lc_mag.push_back(dt.real("magnitude"));
        S.lc_magerr.push_back(dt.real("magnitude error"));
    }
    std::string extra;
    if (dt.next(extra)) tk.fail("lightcurve data file " + S.lcname + " has more than the points listed");
    if (np < 0) {
        // the sorted distinct observation epochs (src/shape/read_dat.c:1990-2004)
        std::vector<double> e = S.lc_t0;
        std::sort(e.begin(), e.end());
        for (size_t i = 0; i < e.size(); i++)
            if (i == 0 || e[i] > e[i - 1]) S.x0.push_back(e[i]);
    }
}

// The '=' state ties a set's value to the last earlier set that gives its
// own: each component of the angle and spin offsets on its own
// (realize_angleoff / realize_omegaoff, src/shape/realize_spin.c:283-337),
// and the whole delay-correction polynomial with its epoch when the first
// coefficient has it (realize_delcor, src/shape/realize_delcor.c:60-146).
// The first set cannot take '='; a tied polynomial must have the earlier
// one's degree and an epoch within half a second of it.
static void tie_obs_sets(std::vector<shape_obs_file::Set> &sets, const Tokens &tk)
{
    constexpr double HALF_SECOND_DAYS = 5.8e-6;
    for (int j = 0; j < 3; j++) {
        int sa = -1, so = -1;
        for (size_t s = 0; s < sets.size(); s++) {
            shape_obs_file::Set &S = sets[s];
            if (S.angle_state[j] != '=') sa = (int)s;
            else if (sa < 0) tk.fail("the first dataset's angle offsets cannot take the = state");
            else S.angleoff[j] = sets[sa].angleoff[j];
            if (S.omega_state[j] != '=') so = (int)s;
            else if (so < 0) tk.fail("the first dataset's spin offsets cannot take the = state");
            else S.omegaoff[j] = sets[so].omegaoff[j];
        }
    }
    int sd = -1;
    for (size_t s = 0; s < sets.size(); s++) {
        shape_obs_file::Set &S = sets[s];
        if (S.lightcurve || S.poset) continue;   // no delay polynomial
        if (S.delcor_state != '=') { sd = (int)s; continue; }
        if (sd < 0) tk.fail("the first delay-correction polynomial cannot take the = state");
        const shape_obs_file::Set &T = sets[sd];
        if (S.delcor.size() != T.delcor.size())
            tk.fail("delay-correction polynomials tied by = must have the same degree");
        if (fabs(S.delcor_t0 - T.delcor_t0) > HALF_SECOND_DAYS)
            tk.fail("delay-correction polynomials tied by = must have the same epoch");
        S.delcor_t0 = T.delcor_t0;
        S.delcor = T.delcor;
    }
}

extern "C" {

// The frames' windows and dof, and the pixel-weighting masks of set s
// (read_deldop / read_doppler, src/shape/read_dat.c:696-762, 1059-1118):
// mask_SS_FF.txt (FFF when the set has more than 100 frames) in the mask
// directory, or the set's data directory without one; ndel x ndop weights
// (ndop for a Doppler set) whose positive entries give the frame's window
// and its dof (the frame's weight per positive entry). A frame without a
// mask keeps the whole image and weight x pixels of dof. A missing mask
// file is an error only when required (shape_obs_set_maskdir); otherwise the
// frame stays unloaded and the set's accessors report it.
static int load_masks(shape_obs_file &o, int s, bool required)
{
    shape_obs_file::Set &S = o.sets[s];
    if (S.lightcurve || S.poset) return SHAPE_OK;
    const int nf = (int)S.frames.size();
    const int nd = S.doppler ? 1 : S.ndel, np = S.ndop;
    const std::string dir = o.maskdir.empty() ? S.dir : o.maskdir;
    for (int f = 0; f < nf; f++) {
        shape_obs_file::Frame &F = S.frames[f];
        F.mask.clear();
        if (!F.weighted) {
            F.win[0] = 1; F.win[1] = nd; F.win[2] = 1; F.win[3] = np;
            F.dof = F.weight * nd * np;
            continue;
        }
        char name[64];
        snprintf(name, sizeof name, nf > 100 ? "mask_%02d_%03d.txt" : "mask_%02d_%02d.txt", s, f);
        const std::string path = dir + "/" + name;
        FILE *fp = fopen(path.c_str(), "rb");
        if (!fp) {
            if (required) return shape::report_error(SHAPE_E_ARG, "obs: cannot open mask file " + path);
            continue;
        }
        std::string text;
        char buf[1 << 16];
        size_t got;
        while ((got = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, got);
        fclose(fp);
        std::vector<double> w;
        try {
            Tokens tk(std::move(text));
            const std::string kind = "mask file " + path;
            tk.set_kind(kind.c_str());
            std::string t;
            while (tk.next(t)) {
                char *end = nullptr;
                const double v = strtod(t.c_str(), &end);
                if (*end != '\0') tk.fail("expected a number (mask weight), got " + t);
                w.push_back(v);
            }
        } catch (const ParseError &e) {
            return shape::report_error(e.code, "obs: " + e.msg);
        }
        if ((long long)w.size() != (long long)nd * np)
            return shape::report_error(SHAPE_E_ARG, "obs: mask file " + path + " holds " + std::to_string(w.size()) +
                                                        " weights, expected " + std::to_string((long long)nd * np));
        int d0 = nd + 1, d1 = 0, p0 = np + 1, p1 = 0;
        double dof = 0.0;
        for (int j = 1; j <= nd; j++)
            for (int k = 1; k <= np; k++)
                if (w[(size_t)(j - 1) * np + (k - 1)] > 0.0) {
                    dof += F.weight;
                    d0 = std::min(d0, j); d1 = std::max(d1, j);
                    p0 = std::min(p0, k); p1 = std::max(p1, k);
                }
        if (d1 < d0) return shape::report_error(SHAPE_E_ARG, "obs: mask file " + path + " has no positive weight");
        F.win[0] = d0; F.win[1] = d1; F.win[2] = p0; F.win[3] = p1;
        F.dof = dof;
        F.mask = std::move(w);
    }
    return SHAPE_OK;
}

// Set s's frames all have their masks (loaded at shape_obs_read or by
// shape_obs_set_maskdir).
static int masks_ready(const shape_obs_file::Set &S, const char *what)
{
    for (const shape_obs_file::Frame &F : S.frames)
        if (F.weighted && F.mask.empty())
            return shape::report_error(SHAPE_E_ARG, std::string(what) + ": the mask of frame " + F.name +
                                                        " was not found (shape_obs_set_maskdir)");
    return SHAPE_OK;
}

int shape_obs_read(const char *path, shape_obs_file **out)
{
    if (!path || !out) return shape::report_error(SHAPE_E_ARG, "obs_read: null argument");
    *out = nullptr;
    FILE *fp = fopen(path, "rb");
    if (!fp) return shape::report_error(SHAPE_E_ARG, std::string("obs_read: cannot open ") + path);
    std::string text;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, fp)) > 0) text.append(buf, got);
    fclose(fp);
    shape_obs_file *o = new shape_obs_file();
    try {
        Tokens tk(std::move(text));
        tk.set_kind("observation file");
        const int nsets = tk.integer("number of datasets");
        if (nsets < 1) tk.fail("no datasets");
        for (int s = 0; s < nsets; s++) {
            shape_obs_file::Set S;
            tk.integer("input node");
            // dataset angle offsets wrapped to [-180, 180) deg, then radians
            // (src/shape/read_dat.c:436-446)
            for (int i = 0; i < 3; i++) {
                double v = tk.param("angle offset", &S.angle_state[i]);
                v += 360.0 * floor((180.0 - v) / 360.0);
                S.angleoff[i] = v * D2R;
            }
            for (int i = 0; i < 3; i++) S.omegaoff[i] = tk.param("spin offset", &S.omega_state[i]) * D2R;
            const std::string type = tk.word("dataset type");
            if (type == "lightcurve" || type == "heliocurve") {
                read_lghtcrv_set(tk, S);
                o->sets.push_back(std::move(S));
                continue;
            }
            if (type == "plane-of-sky") {
                read_poset_set(tk, S);
                o->sets.push_back(std::move(S));
                continue;
            }
            if (type != "delay-doppler" && type != "doppler")
                tk.fail("dataset type " + type + " is not supported", SHAPE_E_UNSUPPORTED);
            S.doppler = type == "doppler";
            // read_deldop / read_doppler headers (src/shape/read_dat.c:528-640, 920-1000)
            S.iradlaw = tk.integer("radar law");
            if (S.iradlaw < 0) tk.fail("negative radar law index");
            const int ne = tk.integer("ephemeris points");
            if (ne < 2) tk.fail("an ephemeris needs at least 2 points");
            for (int i = 0; i < ne; i++) {
                shape_ephem_point e;
                e.t = read_epoch(tk, "ephemeris epoch");
                e.ra = tk.real("RA") * D2R;
                e.dec = tk.real("Dec") * D2R;
                e.dist = tk.real("distance");
                S.ephem.push_back(e);
            }
            memset(&S.dd, 0, sizeof S.dd);
            S.dd.Ftx = tk.real("Ftx");
            if (S.doppler) {
                S.ndel = 1;
                S.ndop = tk.integer("Doppler bins");
                S.dd.dop_per_pixel = tk.real("Doppler bin width");
                S.dopcom = tk.real("Doppler COM bin");
                S.dd.del_per_pixel = 1.0;
                S.dd.spb = S.dd.stride = 1;
                S.dd.codemethod = SHAPE_CODE_LONG_ORIG;
            } else {
            S.ndel = tk.integer("delay bins");
            S.dd.del_per_pixel = tk.real("delay resolution");
            S.dd.spb = tk.integer("samples per baud");
            S.dd.stride = tk.integer("stride");
            if (S.dd.spb < 1 || S.dd.stride < 1 || S.dd.spb % S.dd.stride != 0)
                tk.fail("stride must divide evenly into spb");
            const std::string code = tk.word("code method");
            if (code == "short") S.dd.codemethod = SHAPE_CODE_SHORT;
            else if (code == "long1" || code == "long_orig") S.dd.codemethod = SHAPE_CODE_LONG_ORIG;
            else if (code == "long2" || code == "long_mod") S.dd.codemethod = SHAPE_CODE_LONG_MOD;
            else tk.fail("code method " + code + " is not known");
            S.ndop = tk.integer("Doppler bins");
            S.dd.dop_per_pixel = tk.real("Doppler resolution");
            S.dopcom = tk.real("Doppler COM bin");
            S.dopDC = tk.real("Doppler DC bin");
            S.dd.dopfftlen = tk.integer("Doppler FFT length");
            }
            S.delcor_t0 = read_epoch(tk, "delay-correction epoch");
            const int nd = tk.integer("delay-correction order");
            if (nd < 0) tk.fail("negative delay-correction order");
            for (int i = 0; i <= nd; i++) {
                char st;
                S.delcor.push_back(tk.param("delay-correction coefficient", &st));
                if (i == 0) S.delcor_state = st;
            }
            S.dd.dopscale = tk.param("dopscale", nullptr);
            const int nviews = tk.integer("views per frame");
            S.view_interval = tk.real("view interval") / 86400.0;
            const std::string smear = tk.word("smearing mode");
            if (smear != "center" && smear != "first") tk.fail("smearing mode " + smear + " is not known");
            if (nviews < 1) tk.fail("views per frame must be >= 1");
            if (nviews != 1 && S.doppler)
                tk.fail("smeared Doppler frames (more than one view) are not supported", SHAPE_E_UNSUPPORTED);
            S.nviews = nviews;
            S.v0 = smear == "center" ? nviews / 2 : 0;
            S.dir = tk.word("data directory");
            const int nf = tk.integer("number of frames");
            if (nf < 1) tk.fail("no frames");
            for (int i = 0; i < nf; i++) {
                shape_obs_file::Frame F;
                F.name = tk.word("data file");
                F.t0 = read_epoch(tk, "frame epoch");
                F.sdev = tk.real("sdev");
                F.cal = tk.param("calibration", &F.cal_state);
                if (F.cal <= 0.0 && F.cal_state == 'c') tk.fail("a fixed calibration must be > 0");
                F.nlooks = tk.real("looks");
                F.delcom = S.doppler ? 1.0 : tk.real("delay COM bin");
                F.weight = tk.real("weight");
                F.weighted = tk.integer("pixel weighting") != 0;
                if (F.name.size() >= 3 && F.name.compare(F.name.size() - 3, 3, ".gz") == 0)
                    tk.fail("gzipped data files are not supported", SHAPE_E_UNSUPPORTED);
                S.frames.push_back(F);
            }
            o->sets.push_back(std::move(S));
        }
        tie_obs_sets(o->sets, tk);
    } catch (const ParseError &e) {
        delete o;
        return shape::report_error(e.code, "obs_read: " + e.msg);
    }
    for (size_t s = 0; s < o->sets.size(); s++) load_masks(*o, (int)s, false);
    *out = o;
    return SHAPE_OK;
}

int shape_obs_set_maskdir(shape_obs_file *o, const char *dir)
{
    if (!o || !dir) return shape::report_error(SHAPE_E_ARG, "obs_set_maskdir: null argument");
    o->maskdir = dir;
    for (size_t s = 0; s < o->sets.size(); s++)
        if (int rc = load_masks(*o, (int)s, true)) return rc;
    return SHAPE_OK;
}

void shape_obs_free(shape_obs_file *o) { delete o; }

int shape_obs_nsets(const shape_obs_file *o) { return o ? (int)o->sets.size() : shape::report_error(SHAPE_E_ARG, "obs_nsets: null argument"); }

int shape_obs_set_type(const shape_obs_file *o, int s)
{
    if (!o || s < 0 || s >= (int)o->sets.size()) return shape::report_error(SHAPE_E_ARG, "obs_set_type: no such set");
    return o->sets[s].poset ? 3 : (o->sets[s].lightcurve ? 2 : o->sets[s].doppler);
}

int shape_obs_set(const shape_obs_file *o, int s, shape_deldop_set *set, int *iradlaw, int *nframes,
                  double angleoff[3], double omegaoff[3], size_t *nelem)
{
    if (!o || s < 0 || s >= (int)o->sets.size()) return shape::report_error(SHAPE_E_ARG, "obs_set: no such set");
    const shape_obs_file::Set &S = o->sets[s];
    if (set) {
        shape_radar_law law = set->law;
        *set = S.dd;
        set->law = law;
    }
    if (iradlaw) *iradlaw = S.iradlaw;
    if (nframes) *nframes = (int)S.frames.size();
    for (int i = 0; i < 3; i++) {
        if (angleoff) angleoff[i] = S.angleoff[i];
        if (omegaoff) omegaoff[i] = S.omegaoff[i];
    }
    if (nelem) {
        // each frame's window of positive mask weights (the whole image
        // without a mask)
        if (int rc = masks_ready(S, "obs_set")) return rc;
        size_t n = 0;
        for (const shape_obs_file::Frame &F : S.frames)
            n += (size_t)(F.win[1] - F.win[0] + 1) * (size_t)(F.win[3] - F.win[2] + 1);
        *nelem = n;
    }
    return SHAPE_OK;
}

int shape_obs_views(const shape_obs_file *o, int s, int *nviews, int *v0)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !nviews)
        return shape::report_error(SHAPE_E_ARG, "obs_views: invalid argument");
    *nviews = o->sets[s].nviews;
    if (v0) *v0 = o->sets[s].v0;
    return SHAPE_OK;
}

// Every view of every frame of delay-Doppler set S (read_deldop,
// src/shape/read_dat.c:860-905; deldopoffs, src/shape/deldopoffs.c:19-45;
// realize_spin, src/shape/realize_spin.c:130-185): view k of frame f (the
// reference's numbering) sits at t0 + (k - v0) * view interval, light-time
// corrected; views[f * nviews + j] receives view (v0 + 1 + j) % nviews, the
// order calc_deldop renders them, so the epoch view v0 closes each frame.
static int obs_deldop_views(const shape_obs_file::Set &S, const shape_spin_state *spin, int pos_n,
                            double km_per_pixel, const shape_obs_options *opt, shape_deldop_frame *views,
                            double *obs, double *oneovervar, double *sdev)
{
    if (int rc = masks_ready(S, "obs_frames")) return rc;
    const int nf = (int)S.frames.size(), nv = S.nviews;
    const size_t N = (size_t)nf * nv;
    size_t off = 0;
    std::vector<double> t(N), orb(3 * N), ae(9 * N), sp(3 * N);
    std::vector<shape_deldop_frame> vk(N);     // reference view order
    for (int f = 0; f < nf; f++) {
        const shape_obs_file::Frame &F = S.frames[f];
        shape_deldop_frame G;
        memset(&G, 0, sizeof G);
        G.pos_n = pos_n;
        G.km_per_pixel = km_per_pixel;
        // the window of the frame's positive mask weights (the whole image
        // without a mask), its COM and DC bins counted from the window
        G.ndel = F.win[1] - F.win[0] + 1;
        G.ndop = F.win[3] - F.win[2] + 1;
        G.delcom_vig = F.delcom - F.win[0] + 1;
        G.dopcom_vig = S.dopcom - F.win[2] + 1;
        G.dopDC_vig = S.dopDC - F.win[2] + 1;
        G.weight = F.weight;
        G.dof = F.dof;
        G.cal_floating = F.cal_state == 'f';
        G.cal = F.cal;
        for (int k = 0; k < nv; k++) {
            const size_t i = (size_t)f * nv + k;
            shape_deldop_frame &V = vk[i];
            V = G;
            const double tk = nv == 1 ? F.t0 : F.t0 + (k - S.v0) * S.view_interval;
            if (int rc = shape_ephem_radar_view(S.ephem.data(), (int)S.ephem.size(), tk, opt->perform_ltc, &t[i],
                                                V.oe, &orb[3 * i]))
                return rc;
            if (int rc = shape_delcor_offsets(S.delcor.data(), (int)S.delcor.size() - 1, S.delcor_t0, t[i],
                                              S.dd.del_per_pixel, S.dd.dop_per_pixel, S.dd.Ftx, &V.deloff,
                                              &V.dopoff))
                return rc;
        }
        if (sdev) sdev[f] = F.sdev;
        const std::string full = S.dir + "/" + F.name;
        const int dl[2] = {F.win[0], F.win[1]}, dp[2] = {F.win[2], F.win[3]};
        if (int rc = shape_read_radar_data(full.c_str(), S.ndel, S.ndop, dl, dp, opt->big_endian, F.sdev,
                                           opt->dd_gamma, opt->speckle ? F.nlooks : 0.0,
                                           F.weighted ? F.mask.data() : nullptr, obs + off, oneovervar + off))
            return rc;
        off += (size_t)G.ndel * G.ndop;
    }
    if (int rc = shape_realize_spin(spin, S.angleoff, S.omegaoff, (int)N, t.data(), orb.data(), ae.data(), sp.data()))
        return rc;
    for (size_t i = 0; i < N; i++) {
        memcpy(vk[i].ae, &ae[9 * i], sizeof vk[i].ae);
        memcpy(vk[i].spin, &sp[3 * i], sizeof vk[i].spin);
    }
    for (int f = 0; f < nf; f++)
        for (int j = 0; j < nv; j++) views[(size_t)f * nv + j] = vk[(size_t)f * nv + (S.v0 + 1 + j) % nv];
    return SHAPE_OK;
}

int shape_obs_frames_views(const shape_obs_file *o, int s, const shape_spin_state *spin, int pos_n,
                           double km_per_pixel, const shape_obs_options *opt, shape_deldop_frame *views, double *obs,
                           double *oneovervar, double *sdev)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !spin || !opt || !views || !obs || !oneovervar)
        return shape::report_error(SHAPE_E_ARG, "obs_frames_views: invalid argument");
    const shape_obs_file::Set &S = o->sets[s];
    if (S.lightcurve || S.doppler || S.poset)
        return shape::report_error(SHAPE_E_ARG, "obs_frames_views: not a delay-Doppler set");
    return obs_deldop_views(S, spin, pos_n, km_per_pixel, opt, views, obs, oneovervar, sdev);
}

int shape_obs_frames(const shape_obs_file *o, int s, const shape_spin_state *spin, int pos_n, double km_per_pixel,
                     const shape_obs_options *opt, shape_deldop_frame *frames, double *obs, double *oneovervar,
                     double *sdev)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !spin || !opt || !frames || !obs || !oneovervar)
        return shape::report_error(SHAPE_E_ARG, "obs_frames: invalid argument");
    const shape_obs_file::Set &S = o->sets[s];
    if (S.lightcurve || S.poset)
        return shape::report_error(SHAPE_E_ARG, "obs_frames: a lightcurve or plane-of-sky set");
    if (S.doppler) return shape::report_error(SHAPE_E_ARG, "obs_frames: a Doppler set (use shape_obs_doppler)");
    if (S.nviews != 1)
        return shape::report_error(SHAPE_E_UNSUPPORTED, "obs_frames: smeared frames (use shape_obs_frames_views)");
    return obs_deldop_views(S, spin, pos_n, km_per_pixel, opt, frames, obs, oneovervar, sdev);
}

// A Doppler set's setup and frames (read_doppler, src/shape/read_dat.c:
// 920-1180; dopoffs, src/shape/dopoffs.c:19-40), as shape_obs_frames does
// for delay-Doppler sets.
int shape_obs_doppler(const shape_obs_file *o, int s, const shape_spin_state *spin, int pos_n, double km_per_pixel,
                      const shape_obs_options *opt, shape_doppler_set *set, shape_doppler_frame *frames, double *obs,
                      double *oneovervar)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !spin || !opt || !set || !frames || !obs || !oneovervar)
        return shape::report_error(SHAPE_E_ARG, "obs_doppler: invalid argument");
    const shape_obs_file::Set &S = o->sets[s];
    if (!S.doppler) return shape::report_error(SHAPE_E_ARG, "obs_doppler: not a Doppler set");
    const shape_radar_law law = set->law;
    memset(set, 0, sizeof *set);
    set->dop_per_bin = S.dd.dop_per_pixel;
    set->Ftx = S.dd.Ftx;
    set->dopscale = S.dd.dopscale;
    set->law = law;
    if (int rc = masks_ready(S, "obs_doppler")) return rc;
    const int nf = (int)S.frames.size();
    size_t off = 0;
    std::vector<double> t(nf), orb(3 * (size_t)nf), ae(9 * (size_t)nf), sp(3 * (size_t)nf);
    for (int f = 0; f < nf; f++) {
        const shape_obs_file::Frame &F = S.frames[f];
        shape_doppler_frame &G = frames[f];
        memset(&G, 0, sizeof G);
        G.pos_n = pos_n;
        G.km_per_pixel = km_per_pixel;
        if (int rc = shape_ephem_radar_view(S.ephem.data(), (int)S.ephem.size(), F.t0, opt->perform_ltc, &t[f],
                                            G.oe, &orb[3 * (size_t)f]))
            return rc;
        double deloff;
        if (int rc = shape_delcor_offsets(S.delcor.data(), (int)S.delcor.size() - 1, S.delcor_t0, t[f], 1.0,
                                          S.dd.dop_per_pixel, S.dd.Ftx, &deloff, &G.dopoff))
            return rc;
        // the window of the frame's positive mask weights (the whole
        // spectrum without a mask), its COM bin counted from the window
        G.ndop = F.win[3] - F.win[2] + 1;
        G.dopcom_vig = S.dopcom - F.win[2] + 1;
        G.weight = F.weight;
        G.dof = F.dof;
        G.cal_floating = F.cal_state == 'f';
        G.cal = F.cal;
        G.sdev = F.sdev;
        const std::string full = S.dir + "/" + F.name;
        const int dl[2] = {1, 1}, dp[2] = {F.win[2], F.win[3]};
        if (int rc = shape_read_radar_data(full.c_str(), 1, S.ndop, dl, dp, opt->big_endian, F.sdev, 1.0,
                                           opt->speckle ? F.nlooks : 0.0, F.weighted ? F.mask.data() : nullptr,
                                           obs + off, oneovervar + off))
            return rc;
        off += (size_t)G.ndop;
    }
    if (int rc = shape_realize_spin(spin, S.angleoff, S.omegaoff, nf, t.data(), orb.data(), ae.data(), sp.data()))
        return rc;
    for (int f = 0; f < nf; f++) {
        memcpy(frames[f].ae, &ae[9 * (size_t)f], sizeof frames[f].ae);
        memcpy(frames[f].spin, &sp[3 * (size_t)f], sizeof frames[f].spin);
    }
    return SHAPE_OK;
}

int shape_obs_lghtcrv_info(const shape_obs_file *o, int s, int *ioptlaw, int *ncalc, int *n)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !o->sets[s].lightcurve)
        return shape::report_error(SHAPE_E_ARG, "obs_lghtcrv_info: not a lightcurve set");
    const shape_obs_file::Set &S = o->sets[s];
    if (ioptlaw) *ioptlaw = S.ioptlaw;
    if (ncalc) *ncalc = (int)S.x0.size();
    if (n) *n = (int)S.lc_t0.size();
    return SHAPE_OK;
}

// A lightcurve set ready for shape_engine_add_lghtcrv_set, as read_lghtcrv
// and realize_spin leave it (src/shape/read_dat.c:1856-1956, 2010-2029;
// src/shape/realize_spin.c:223-260): each calculated epoch light-time
// corrected through the ephemerides (x = x0 - DAYSPERAU * distance, the
// view taken again there), its observer and Sun matrices and solar phase,
// its body matrix from the spin state with the set's angle and spin
// offsets; each observation's magnitude turned into an intensity relative
// to the Sun's (sun_appmag, the .par file's value for this set's optical
// law) and its epoch light-time corrected the same way.
int shape_obs_poset_info(const shape_obs_file *o, int s, int *ioptlaw, int *nframes)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !o->sets[s].poset || !ioptlaw || !nframes)
        return shape::report_error(SHAPE_E_ARG, "obs_poset_info: not a plane-of-sky set");
    *ioptlaw = o->sets[s].ioptlaw;
    *nframes = (int)o->sets[s].pframes.size();
    return SHAPE_OK;
}

int shape_obs_poset_file(const shape_obs_file *o, int s, int frame, char *path, int size, int *pixels_weighted)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !o->sets[s].poset || !path || size < 1 ||
        frame < 0 || frame >= (int)o->sets[s].pframes.size())
        return shape::report_error(SHAPE_E_ARG, "obs_poset_file: invalid argument");
    const shape_obs_file::Set &S = o->sets[s];
    const std::string full = S.dir + "/" + S.pframes[frame].name;
    if ((int)full.size() >= size) return shape::report_error(SHAPE_E_ARG, "obs_poset_file: buffer too small");
    memcpy(path, full.c_str(), full.size() + 1);
    if (pixels_weighted) *pixels_weighted = S.pframes[frame].pixels_weighted;
    return SHAPE_OK;
}

// read_poset's views (src/shape/read_dat.c:1520-1560) for one view per frame:
// ephem2mat at the frame epoch, with light-time correction when asked (the
// fit grid's km per pixel takes the distance before the correction, as
// read_poset's does), then the spin realized at the corrected epochs.
int shape_obs_poset(const shape_obs_file *o, int s, const shape_spin_state *spin, const shape_obs_options *opt,
                    shape_poset_frame *frames)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !o->sets[s].poset || !spin || !opt || !frames)
        return shape::report_error(SHAPE_E_ARG, "obs_poset: invalid argument");
    const shape_obs_file::Set &S = o->sets[s];
    if (S.nviews != 1)
        return shape::report_error(SHAPE_E_UNSUPPORTED, "obs_poset: smeared plane-of-sky frames");
    const double DAYSPERAU = 5.775518328e-3;   // src/shape/const.h:144
    const double AU = 1.4959787061e8;         // km (src/shape/const.h:135)
    const int nf = (int)S.pframes.size();
    const shape_ephem_point *A = S.ephem.data(), *U = S.solephem.data();
    const int na = (int)S.ephem.size(), nu = (int)S.solephem.size();
    std::vector<double> t(nf), orb(3 * (size_t)nf), ae(9 * (size_t)nf), sp(3 * (size_t)nf);
    for (int i = 0; i < nf; i++) {
        shape_poset_frame &F = frames[i];
        const shape_obs_file::Set::PosFrame &R = S.pframes[i];
        double az, dist, dist1;
        t[i] = R.t0;
        if (int rc = shape_ephem_view(A, na, U, nu, t[i], F.oe, F.se, &orb[3 * (size_t)i], &F.solar_phase, &az, &dist))
            return rc;
        if (opt->perform_ltc) {
            t[i] -= DAYSPERAU * dist;
            if (int rc = shape_ephem_view(A, na, U, nu, t[i], F.oe, F.se, &orb[3 * (size_t)i], &F.solar_phase, &az,
                                          &dist1))
                return rc;
        }
        F.fit_km_per_pixel = S.angle_per_pixel * (dist * AU);
        F.northangle = R.northangle;
        F.xoff = R.off[0];
        F.yoff = R.off[1];
        F.weight = R.weight;
    }
    if (int rc = shape_realize_spin(spin, S.angleoff, S.omegaoff, nf, t.data(), orb.data(), ae.data(), sp.data()))
        return rc;
    for (int i = 0; i < nf; i++) memcpy(frames[i].ae, &ae[9 * (size_t)i], sizeof frames[i].ae);
    return SHAPE_OK;
}

int shape_obs_lghtcrv(const shape_obs_file *o, int s, const shape_spin_state *spin, int pos_n, double km_per_pixel,
                      const shape_obs_options *opt, double sun_appmag, shape_lghtcrv_set *set,
                      shape_lghtcrv_point *points, double *x, double *t, double *obs, double *oneovervar)
{
    if (!o || s < 0 || s >= (int)o->sets.size() || !o->sets[s].lightcurve || !spin || !opt || !set || !points ||
        !x || !t || !obs || !oneovervar)
        return shape::report_error(SHAPE_E_ARG, "obs_lghtcrv: invalid argument");
    const shape_obs_file::Set &S = o->sets[s];
    const double DAYSPERAU = 5.775518328e-3;   // src/shape/const.h:144
    const double LN10 = 2.302585092994046;     // src/shape/const.h:133
    const int nc = (int)S.x0.size(), n = (int)S.lc_t0.size();
    const shape_ephem_point *A = S.ephem.data(), *U = S.solephem.data();
    const int na = (int)S.ephem.size(), nu = (int)S.solephem.size();
    std::vector<double> orb(3 * (size_t)nc), ae(9 * (size_t)nc), sp(3 * (size_t)nc);
    for (int i = 0; i < nc; i++) {
        shape_lghtcrv_point &P = points[i];
        memset(&P, 0, sizeof P);
        P.pos_n = pos_n;
        P.km_per_pixel = km_per_pixel;
        double az, dist;
        x[i] = S.x0[i];
        if (int rc = shape_ephem_view(A, na, U, nu, x[i], P.oe, P.se, &orb[3 * (size_t)i], &P.solar_phase, &az, &dist))
            return rc;
        if (opt->perform_ltc) {
            x[i] = S.x0[i] - DAYSPERAU * dist;
            if (int rc = shape_ephem_view(A, na, U, nu, x[i], P.oe, P.se, &orb[3 * (size_t)i], &P.solar_phase, &az,
                                          &dist))
                return rc;
        }
    }
    for (int i = 0; i < n; i++) {
        const double intens = exp(-0.4 * LN10 * (S.lc_mag[i] - sun_appmag));
        const double err = (0.4 * LN10 * S.lc_magerr[i]) * intens;
        obs[i] = intens;
        oneovervar[i] = 1.0 / (err * err);
        t[i] = S.lc_t0[i];
        if (opt->perform_ltc) {
            double oe[9], se[9], os[3], ph, az, dist;
            if (int rc = shape_ephem_view(A, na, U, nu, t[i], oe, se, os, &ph, &az, &dist)) return rc;
            t[i] -= DAYSPERAU * dist;
        }
    }
    if (int rc = shape_realize_spin(spin, S.angleoff, S.omegaoff, nc, x, orb.data(), ae.data(), sp.data()))
        return rc;
    for (int i = 0; i < nc; i++) memcpy(points[i].ae, &ae[9 * (size_t)i], sizeof points[i].ae);
    shape_optical_law law = set->law;
    memset(set, 0, sizeof *set);
    set->law = law;
    set->ncalc = nc;
    set->n = n;
    set->x = x;
    set->t = t;
    set->obs = obs;
    set->oneovervar = oneovervar;
    set->weight = S.lc_weight;
    set->dof = S.lc_weight * n;
    set->cal_floating = S.lc_cal_state == 'f';
    set->cal = S.lc_cal;
    return SHAPE_OK;
}

// The listfit output of a radar frame (src/shape/chi2.c:555-558): one line
// "%13.6e" of cal * fit / sdev per bin, delay-major.
int shape_write_fitdat(const char *path, int ndel, int ndop, const double *fit, double cal, double sdev)
{
    if (!path || !fit || ndel < 1 || ndop < 1) return shape::report_error(SHAPE_E_ARG, "write_fitdat: invalid argument");
    FILE *fp = fopen(path, "w");
    if (!fp) return shape::report_error(SHAPE_E_ARG, std::string("write_fitdat: cannot create ") + path);
    for (size_t k = 0; k < (size_t)ndel * ndop; k++) fprintf(fp, "%13.6e\n", cal * fit[k] / sdev);
    const int bad = ferror(fp);
    if (fclose(fp) != 0 || bad) return shape::report_error(SHAPE_E_ARG, std::string("write_fitdat: write failed: ") + path);
    return SHAPE_OK;
}

}  // extern "C"
