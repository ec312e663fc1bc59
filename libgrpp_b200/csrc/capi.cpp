// libgrpp C API on top of the B200 engine.
//
// Containers keep libgrpp's semantics (libgrpp/shell.c, potential.c, grpp.c,
// parameters.c). Every integrator builds a one-task batch and runs the same
// GPU pipeline as the batched entry points (engine.cu). Differences from the
// reference's behaviour, by design:
//  * no caller object is written during a call (libgrpp binds the outercore
//    shells' origins to the centre, libgrpp/outercore_integrals.c:107-111, which
//    makes concurrent calls on one GRPP object race); the result is the same;
//  * misuse is reported through libgrpp_b200_last_error() with the outputs
//    zeroed, instead of assert().
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/libgrpp.h"
#include "../../include/libgrpp_b200.h"
#include "engine.h"
#include "nucmodel.h"
#include "tables.h"

namespace {

int gen_dirac(int L, int *cl)
{
    int c = 0;
    for (int r = L; r >= 0; r--)
        for (int s = L; s >= 0; s--)
            for (int t = L; t >= 0; t--)
                if (r + s + t == L) {
                    cl[3 * c] = r;
                    cl[3 * c + 1] = s;
                    cl[3 * c + 2] = t;
                    c++;
                }
    return (L + 1) * (L + 2) / 2;
}

int gen_turbomole(int L, int *cl)
{
    int c = 0;
    for (int r = L; r >= 0; r--)
        for (int s = L - r; s >= 0; s--) {
            cl[3 * c] = r;
            cl[3 * c + 1] = s;
            cl[3 * c + 2] = L - r - s;
            c++;
        }
    return (L + 1) * (L + 2) / 2;
}

int g_initialized = 0;
std::mutex g_init_mu;

constexpr int kMaxPots = 100;  // grpp.c:12

double gaussian_norm(int L, double a) { return std::pow(2 * a / M_PI, 0.75) * std::pow(4 * a, 0.5 * L); }

int ncart_h(int L) { return (L + 1) * (L + 2) / 2; }

// Flat batch assembled from libgrpp objects.
struct Builder {
    std::vector<int> shell_L, shell_nprim, shell_prim_off, shell_cart_off, cart_list;
    std::vector<double> prim_coef, prim_alpha, shell_origin;
    std::vector<int> pot_L, pot_J, pot_nprim, pot_prim_off, pot_powers;
    std::vector<double> pot_coef, pot_alpha;
    std::vector<int> grpp_UL, grpp_arep_off, grpp_n_arep, grpp_so_off, grpp_n_so, grpp_oc_off, grpp_n_oc, grpp_pot_list,
        grpp_oc_pot, grpp_oc_shell;
    std::vector<double> centre_origin;
    std::vector<int> centre_grpp, task_a, task_b, task_c;

    int add_shell(const libgrpp_shell_t *s)
    {
        shell_L.push_back(s->L);
        shell_nprim.push_back(s->num_primitives);
        shell_prim_off.push_back((int)prim_coef.size());
        shell_cart_off.push_back((int)cart_list.size() / 3);
        for (int i = 0; i < 3 * s->cart_size; i++) cart_list.push_back(s->cart_list[i]);
        for (int i = 0; i < s->num_primitives; i++) {
            prim_coef.push_back(s->coeffs[i]);
            prim_alpha.push_back(s->alpha[i]);
        }
        for (int d = 0; d < 3; d++) shell_origin.push_back(s->origin[d]);
        return (int)shell_L.size() - 1;
    }
    int add_pot(const libgrpp_potential_t *p)
    {
        pot_L.push_back(p->L);
        pot_J.push_back(p->J);
        pot_nprim.push_back(p->num_primitives);
        pot_prim_off.push_back((int)pot_coef.size());
        for (int i = 0; i < p->num_primitives; i++) {
            pot_powers.push_back(p->powers[i]);
            pot_coef.push_back(p->coeffs[i]);
            pot_alpha.push_back(p->alpha[i]);
        }
        return (int)pot_L.size() - 1;
    }
    int add_grpp(const libgrpp_potential_t *UL, int n_arep, libgrpp_potential_t *const *arep, int n_so,
                 libgrpp_potential_t *const *so, int n_oc, libgrpp_potential_t *const *ocp, libgrpp_shell_t *const *ocs)
    {
        grpp_UL.push_back(UL ? add_pot(UL) : -1);
        grpp_arep_off.push_back((int)grpp_pot_list.size());
        grpp_n_arep.push_back(n_arep);
        for (int i = 0; i < n_arep; i++) grpp_pot_list.push_back(add_pot(arep[i]));
        grpp_so_off.push_back((int)grpp_pot_list.size());
        grpp_n_so.push_back(n_so);
        for (int i = 0; i < n_so; i++) grpp_pot_list.push_back(add_pot(so[i]));
        grpp_oc_off.push_back((int)grpp_oc_pot.size());
        grpp_n_oc.push_back(n_oc);
        for (int i = 0; i < n_oc; i++) {
            const int p = add_pot(ocp[i]);
            const int s = add_shell(ocs[i]);
            grpp_oc_pot.push_back(p);
            grpp_oc_shell.push_back(s);
        }
        return (int)grpp_UL.size() - 1;
    }
    int add_centre(const double *C, int g)
    {
        for (int d = 0; d < 3; d++) centre_origin.push_back(C[d]);
        centre_grpp.push_back(g);
        return (int)centre_grpp.size() - 1;
    }
    void add_task(int a, int b, int c)
    {
        task_a.push_back(a);
        task_b.push_back(b);
        task_c.push_back(c);
    }
    libgrpp_b200_batch_t view() const
    {
        libgrpp_b200_batch_t v;
        v.n_shells = (int)shell_L.size();
        v.shell_L = shell_L.data();
        v.shell_nprim = shell_nprim.data();
        v.shell_prim_off = shell_prim_off.data();
        v.prim_coef = prim_coef.data();
        v.prim_alpha = prim_alpha.data();
        v.shell_origin = shell_origin.data();
        v.shell_cart_off = shell_cart_off.data();
        v.cart_list = cart_list.data();
        v.n_pots = (int)pot_L.size();
        v.pot_L = pot_L.data();
        v.pot_J = pot_J.data();
        v.pot_nprim = pot_nprim.data();
        v.pot_prim_off = pot_prim_off.data();
        v.pot_powers = pot_powers.data();
        v.pot_coef = pot_coef.data();
        v.pot_alpha = pot_alpha.data();
        v.n_grpps = (int)grpp_UL.size();
        v.grpp_UL = grpp_UL.data();
        v.grpp_arep_off = grpp_arep_off.data();
        v.grpp_n_arep = grpp_n_arep.data();
        v.grpp_so_off = grpp_so_off.data();
        v.grpp_n_so = grpp_n_so.data();
        v.grpp_oc_off = grpp_oc_off.data();
        v.grpp_n_oc = grpp_n_oc.data();
        v.grpp_pot_list = grpp_pot_list.data();
        v.grpp_oc_pot = grpp_oc_pot.data();
        v.grpp_oc_shell = grpp_oc_shell.data();
        v.n_centres = (int)centre_grpp.size();
        v.centre_origin = centre_origin.data();
        v.centre_grpp = centre_grpp.data();
        v.n_tasks = (int64_t)task_a.size();
        v.task_a = task_a.data();
        v.task_b = task_b.data();
        v.task_c = task_c.data();
        return v;
    }
};

bool check_init()
{
    if (!g_initialized) {
        grpp::set_error(LIBGRPP_B200_ERR_NOT_INIT, "libgrpp_init() was not called");
        return false;
    }
    return true;
}

// one shell pair through the one-electron batch (kind 0 overlap, 1 kinetic, 2 momentum)
void onee_single(libgrpp_shell_t *A, libgrpp_shell_t *B, int kind, double *o0, double *o1, double *o2)
{
    const int n = A->cart_size * B->cart_size;
    double *outs[3] = {o0, o1, o2};
    for (double *o : outs)
        if (o) memset(o, 0, n * sizeof(double));
    if (!check_init()) return;
    Builder bd;
    const int ia = bd.add_shell(A), ib = bd.add_shell(B);
    bd.add_task(ia, ib, 0);
    libgrpp_b200_batch_t v = bd.view();
    std::vector<double> tmp[3];
    for (auto &x : tmp) x.assign(n, 0.0);
    if (grpp::run_onee_batch(&v, kind, tmp[0].data(), tmp[1].data(), tmp[2].data()) == 0)
        for (int k = 0; k < 3; k++)
            if (outs[k]) memcpy(outs[k], tmp[k].data(), n * sizeof(double));
}

// run a one-centre batch; out[k] receive consecutive task blocks
int run(const Builder &bd, int raw_so, std::vector<double> out[4])
{
    libgrpp_b200_batch_t v = bd.view();
    const int64_t n = grpp::batch_output_size(&v);
    for (int k = 0; k < 4; k++) out[k].assign(std::max<int64_t>(n, 1), 0.0);
    grpp::RunOptions opt;
    opt.raw_so = raw_so;
    return grpp::run_full_batch(&v, opt, out[0].data(), out[1].data(), out[2].data(), out[3].data());
}

// differentiate_shell (libgrpp/diff_gaussian.c:35-63): L-1 with N_L/N_{L-1}, L+1 with 2 a N_L/N_{L+1}
libgrpp_shell_t *shell_down(const libgrpp_shell_t *s)
{
    if (s->L == 0) return nullptr;
    libgrpp_shell_t *d = libgrpp_new_shell((double *)s->origin, s->L - 1, s->num_primitives, s->coeffs, s->alpha);
    for (int i = 0; i < s->num_primitives; i++)
        d->coeffs[i] *= gaussian_norm(s->L, s->alpha[i]) / gaussian_norm(s->L - 1, s->alpha[i]);
    return d;
}

libgrpp_shell_t *shell_up(const libgrpp_shell_t *s)
{
    libgrpp_shell_t *u = libgrpp_new_shell((double *)s->origin, s->L + 1, s->num_primitives, s->coeffs, s->alpha);
    for (int i = 0; i < s->num_primitives; i++)
        u->coeffs[i] *= 2.0 * s->alpha[i] * gaussian_norm(s->L, s->alpha[i]) / gaussian_norm(s->L + 1, s->alpha[i]);
    return u;
}

// overlap_gradient.c:219-241
int nlm_to_linear(const int *nlm)
{
    const int L = nlm[0] + nlm[1] + nlm[2], n = (L + 1) * (L + 2) / 2;
    std::vector<int> cl(3 * n);
    libgrpp_params.cartesian_generator(L, cl.data());
    int idx;
    for (idx = 0; idx < n; idx++)
        if (cl[3 * idx] == nlm[0] && cl[3 * idx + 1] == nlm[1] && cl[3 * idx + 2] == nlm[2]) break;
    return idx;
}

int points_equal(const double *a, const double *b)
{
    return std::fabs(a[0] - b[0]) < 1e-12 && std::fabs(a[1] - b[1]) < 1e-12 && std::fabs(a[2] - b[2]) < 1e-12;
}

struct GradContribution {
    int diff_bra;
    double factor;
};

// grpp_integrals_gradient.c:280-393: which (differentiated side, sign) terms contribute
std::vector<GradContribution> gradient_terms(const double *A, const double *B, const double *C, const double *D)
{
    std::vector<GradContribution> out;
    if (points_equal(A, C) && points_equal(B, C)) return out;
    if (!points_equal(A, D) && !points_equal(B, D) && !points_equal(C, D)) return out;
    if (!points_equal(A, C) && !points_equal(C, B) && !points_equal(A, B)) {
        if (points_equal(A, D)) out.push_back({1, +1.0});
        if (points_equal(B, D)) out.push_back({0, +1.0});
        if (points_equal(C, D)) {
            out.push_back({1, -1.0});
            out.push_back({0, -1.0});
        }
    }
    if (points_equal(A, B) && !points_equal(A, C)) {
        const double f = points_equal(A, D) ? +1.0 : -1.0;
        out.push_back({1, f});
        out.push_back({0, f});
    }
    if (!points_equal(A, C) && points_equal(C, B)) out.push_back({1, points_equal(A, D) ? +1.0 : -1.0});
    if (points_equal(A, C) && !points_equal(C, B)) out.push_back({0, points_equal(B, D) ? +1.0 : -1.0});
    return out;
}

// Full-GRPP gradient of one shell pair w.r.t. point D for one GRPP description added by add_grpp_fn.
template <typename AddGrpp>
void gradient_impl(libgrpp_shell_t *A, libgrpp_shell_t *B, const double *C, const double *D, AddGrpp add_grpp, int raw_so,
                   double **g0, double **g1, double **g2, double **g3)
{
    const int nA = A->cart_size, nB = B->cart_size, n = nA * nB;
    double **gr[4] = {g0, g1, g2, g3};
    for (int c = 0; c < 4; c++)
        for (int k = 0; k < 3; k++)
            if (gr[c] && gr[c][k]) memset(gr[c][k], 0, n * sizeof(double));
    if (!check_init()) return;
    const std::vector<GradContribution> terms = gradient_terms(A->origin, B->origin, C, D);
    if (terms.empty()) return;
    libgrpp_shell_t *Ad = shell_down(A), *Au = shell_up(A), *Bd = shell_down(B), *Bu = shell_up(B);
    Builder bd;
    const int iA = bd.add_shell(A), iB = bd.add_shell(B), iAu = bd.add_shell(Au), iBu = bd.add_shell(Bu);
    const int iAd = Ad ? bd.add_shell(Ad) : -1, iBd = Bd ? bd.add_shell(Bd) : -1;
    const int g = add_grpp(bd);
    const int c = bd.add_centre(C, g);
    // tasks: (Ad,B) (Au,B) (A,Bd) (A,Bu)
    int t_ad = -1, t_au, t_bd = -1, t_bu, nt = 0;
    std::vector<int64_t> off;
    auto add = [&](int a, int b) {
        bd.add_task(a, b, c);
        return nt++;
    };
    if (iAd >= 0) t_ad = add(iAd, iB);
    t_au = add(iAu, iB);
    if (iBd >= 0) t_bd = add(iA, iBd);
    t_bu = add(iA, iBu);
    std::vector<double> out[4];
    if (run(bd, raw_so, out) == 0) {
        std::vector<int64_t> boff(nt + 1, 0);
        for (int t = 0; t < nt; t++)
            boff[t + 1] = boff[t] + (int64_t)((bd.shell_L[bd.task_a[t]] + 1) * (bd.shell_L[bd.task_a[t]] + 2) / 2) *
                                        ((bd.shell_L[bd.task_b[t]] + 1) * (bd.shell_L[bd.task_b[t]] + 2) / 2);
        for (const GradContribution &tc : terms) {
            const int diff_bra = tc.diff_bra;
            const int td = diff_bra ? t_ad : t_bd, tu = diff_bra ? t_au : t_bu;
            const int nd = diff_bra ? (Ad ? Ad->cart_size : 0) : (Bd ? Bd->cart_size : 0);
            const int nu = diff_bra ? Au->cart_size : Bu->cart_size;
            for (int k = 0; k < 3; k++)
                for (int i = 0; i < nA; i++)
                    for (int j = 0; j < nB; j++) {
                        int bra[3] = {A->cart_list[3 * i], A->cart_list[3 * i + 1], A->cart_list[3 * i + 2]};
                        int ket[3] = {B->cart_list[3 * j], B->cart_list[3 * j + 1], B->cart_list[3 * j + 2]};
                        int *dn = diff_bra ? bra : ket;
                        const int idx = i * nB + j;
                        // libgrpp also forms this term when the exponent is 0, reading outside the
                        // L-1 block and multiplying by 0 (grpp_integrals_gradient.c:452-466);
                        // skipping it gives the same value without the out-of-bounds read
                        if (nd > 0 && dn[k] > 0) {
                            dn[k] -= 1;
                            const int bi = nlm_to_linear(bra), ki = nlm_to_linear(ket);
                            dn[k] += 1;
                            const int nn = dn[k], row = diff_bra ? nB : nd, id = row * bi + ki;
                            for (int cmp = 0; cmp < 4; cmp++)
                                if (gr[cmp]) gr[cmp][k][idx] -= tc.factor * nn * out[cmp][boff[td] + id];
                        }
                        dn[k] += 1;
                        const int bi = nlm_to_linear(bra), ki = nlm_to_linear(ket);
                        dn[k] -= 1;
                        const int row = diff_bra ? nB : nu, id = row * bi + ki;
                        for (int cmp = 0; cmp < 4; cmp++)
                            if (gr[cmp]) gr[cmp][k][idx] += tc.factor * out[cmp][boff[tu] + id];
                    }
        }
    }
    if (Ad) libgrpp_delete_shell(Ad);
    if (Bd) libgrpp_delete_shell(Bd);
    libgrpp_delete_shell(Au);
    libgrpp_delete_shell(Bu);
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

// ============================================================ parameters (parameters.c:17-134)
libgrpp_parameters_t libgrpp_params = {1e-16, 1e-16, 1e-16, gen_dirac};

void libgrpp_set_default_parameters(void)
{
    libgrpp_params.radial_tolerance = 1e-16;
    libgrpp_params.angular_screening_tolerance = 1e-16;
    libgrpp_params.modified_bessel_tolerance = 1e-16;
    libgrpp_params.cartesian_generator = gen_dirac;
}
void libgrpp_set_radial_tolerance(double t) { libgrpp_params.radial_tolerance = t; }
void libgrpp_set_angular_screening_tolerance(double t) { libgrpp_params.angular_screening_tolerance = t; }
void libgrpp_set_modified_bessel_tolerance(double t) { libgrpp_params.modified_bessel_tolerance = t; }
void libgrpp_set_cartesian_order(int order)
{
    if (order == LIBGRPP_CART_ORDER_DIRAC) libgrpp_params.cartesian_generator = gen_dirac;
    else if (order == LIBGRPP_CART_ORDER_TURBOMOLE) libgrpp_params.cartesian_generator = gen_turbomole;
    else grpp::set_error(LIBGRPP_B200_ERR_INVALID, "unknown Cartesian order");
}
void libgrpp_set_cartesian_generator(int (*g)(int, int *)) { libgrpp_params.cartesian_generator = g; }

// ============================================================ init (init_finalize.c:19-50)
void libgrpp_init(void)
{
    std::lock_guard<std::mutex> lk(g_init_mu);
    g_initialized = 1;
}
void libgrpp_finalize(void)
{
    std::lock_guard<std::mutex> lk(g_init_mu);
    g_initialized = 0;
}
int libgrpp_is_initialized(void) { return g_initialized; }

// ============================================================ potentials (potential.c:22-115)
libgrpp_potential_t *libgrpp_new_potential(int L, int J, int n, int *powers, double *coeffs, double *alpha)
{
    libgrpp_potential_t *p = (libgrpp_potential_t *)calloc(1, sizeof(libgrpp_potential_t));
    p->L = L;
    p->J = J;
    p->powers = (int *)calloc(n > 0 ? n : 1, sizeof(int));
    p->coeffs = (double *)calloc(n > 0 ? n : 1, sizeof(double));
    p->alpha = (double *)calloc(n > 0 ? n : 1, sizeof(double));
    for (int i = 0; i < n; i++) {
        if (std::fabs(coeffs[i]) < LIBGRPP_ZERO_THRESH) continue;
        p->coeffs[p->num_primitives] = coeffs[i];
        p->powers[p->num_primitives] = powers[i];
        p->alpha[p->num_primitives] = alpha[i];
        p->num_primitives++;
    }
    return p;
}

void libgrpp_delete_potential(libgrpp_potential_t *p)
{
    if (!p) return;
    free(p->powers);
    free(p->coeffs);
    free(p->alpha);
    free(p);
}

double libgrpp_potential_value(libgrpp_potential_t *p, double r)
{
    double v = 0.0;
    const double r2 = r * r;
    for (int i = 0; i < p->num_primitives; i++) v += p->coeffs[i] * std::pow(r, p->powers[i] - 2) * std::exp(-p->alpha[i] * r2);
    return v;
}

libgrpp_potential_t *libgrpp_shrink_potential(libgrpp_potential_t *src)
{
    const int n = src->num_primitives;
    std::vector<int> pw;
    std::vector<double> c, a;
    for (int i = 0; i < n; i++)
        if (std::fabs(src->coeffs[i]) > LIBGRPP_ZERO_THRESH) {
            pw.push_back(src->powers[i]);
            c.push_back(src->coeffs[i]);
            a.push_back(src->alpha[i]);
        }
    return libgrpp_new_potential(src->L, src->J, (int)c.size(), pw.data(), c.data(), a.data());
}

// ============================================================ shells (shell.c:23-126)
int *libgrpp_generate_shell_cartesians(int L)
{
    const int n = (L + 1) * (L + 2) / 2;
    int *cl = (int *)calloc(3 * n, sizeof(int));
    libgrpp_params.cartesian_generator(L, cl);
    return cl;
}

libgrpp_shell_t *libgrpp_new_shell(double *origin, int L, int n, double *coeffs, double *alpha)
{
    libgrpp_shell_t *s = (libgrpp_shell_t *)malloc(sizeof(libgrpp_shell_t));
    s->L = L;
    for (int d = 0; d < 3; d++) s->origin[d] = origin[d];
    s->cart_size = (L + 1) * (L + 2) / 2;
    s->cart_list = libgrpp_generate_shell_cartesians(L);
    s->num_primitives = n;
    s->coeffs = (double *)calloc(n > 0 ? n : 1, sizeof(double));
    s->alpha = (double *)calloc(n > 0 ? n : 1, sizeof(double));
    for (int i = 0; i < n; i++) {
        s->coeffs[i] = coeffs[i];
        s->alpha[i] = alpha[i];
    }
    return s;
}

libgrpp_shell_t *libgrpp_shell_deep_copy(libgrpp_shell_t *s)
{
    return libgrpp_new_shell(s->origin, s->L, s->num_primitives, s->coeffs, s->alpha);
}

void libgrpp_shell_shrink(libgrpp_shell_t *s)
{
    int n = 0;
    for (int i = 0; i < s->num_primitives; i++)
        if (std::fabs(s->coeffs[i]) > LIBGRPP_ZERO_THRESH) {
            s->coeffs[n] = s->coeffs[i];
            s->alpha[n] = s->alpha[i];
            n++;
        }
    s->num_primitives = n;
}

void libgrpp_shell_mult_normcoef(libgrpp_shell_t *s)
{
    for (int i = 0; i < s->num_primitives; i++) s->coeffs[i] *= gaussian_norm(s->L, s->alpha[i]);
}

int libgrpp_get_shell_size(libgrpp_shell_t *s) { return s->cart_size; }

void libgrpp_delete_shell(libgrpp_shell_t *s)
{
    if (!s) return;
    free(s->cart_list);
    free(s->coeffs);
    free(s->alpha);
    free(s);
}

// ============================================================ GRPP (grpp.c:15-109)
libgrpp_grpp_t *libgrpp_new_grpp(void) { return (libgrpp_grpp_t *)calloc(1, sizeof(libgrpp_grpp_t)); }

void libgrpp_grpp_set_local_potential(libgrpp_grpp_t *g, libgrpp_potential_t *p)
{
    if (g->U_L) libgrpp_delete_potential(g->U_L);
    g->U_L = p;
}

void libgrpp_grpp_add_averaged_potential(libgrpp_grpp_t *g, libgrpp_potential_t *p)
{
    if (g->n_arep == 0) g->U_arep = (libgrpp_potential_t **)calloc(kMaxPots, sizeof(void *));
    if (g->n_arep >= kMaxPots) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, "more than 100 averaged potentials");
        return;
    }
    g->U_arep[g->n_arep++] = p;
}

void libgrpp_grpp_add_spin_orbit_potential(libgrpp_grpp_t *g, libgrpp_potential_t *p)
{
    if (g->n_esop == 0) g->U_esop = (libgrpp_potential_t **)calloc(kMaxPots, sizeof(void *));
    if (g->n_esop >= kMaxPots) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, "more than 100 spin-orbit potentials");
        return;
    }
    g->U_esop[g->n_esop++] = p;
}

void libgrpp_grpp_add_outercore_potential(libgrpp_grpp_t *g, libgrpp_potential_t *p, libgrpp_shell_t *s)
{
    if (g->n_oc_shells == 0) {
        g->U_oc = (libgrpp_potential_t **)calloc(kMaxPots, sizeof(void *));
        g->oc_shells = (libgrpp_shell_t **)calloc(kMaxPots, sizeof(void *));
    }
    if (g->n_oc_shells >= kMaxPots) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, "more than 100 outercore shells");
        return;
    }
    g->U_oc[g->n_oc_shells] = p;
    g->oc_shells[g->n_oc_shells] = s;
    g->n_oc_shells++;
}

void libgrpp_delete_grpp(libgrpp_grpp_t *g)
{
    if (!g) return;
    if (g->U_L) libgrpp_delete_potential(g->U_L);
    for (int i = 0; i < g->n_arep; i++) libgrpp_delete_potential(g->U_arep[i]);
    free(g->U_arep);
    for (int i = 0; i < g->n_esop; i++) libgrpp_delete_potential(g->U_esop[i]);
    free(g->U_esop);
    for (int i = 0; i < g->n_oc_shells; i++) {
        libgrpp_delete_potential(g->U_oc[i]);
        libgrpp_delete_shell(g->oc_shells[i]);
    }
    free(g->U_oc);
    free(g->oc_shells);
    free(g);
}

// ============================================================ integrators
static void one_task(libgrpp_shell_t *A, libgrpp_shell_t *B, const double *C, const libgrpp_potential_t *UL, int n_arep,
                     libgrpp_potential_t *const *arep, int n_so, libgrpp_potential_t *const *so, int n_oc,
                     libgrpp_potential_t *const *ocp, libgrpp_shell_t *const *ocs, int raw_so, double *o0, double *o1,
                     double *o2, double *o3)
{
    const size_t n = (size_t)A->cart_size * B->cart_size;
    double *outs[4] = {o0, o1, o2, o3};
    for (double *o : outs)
        if (o) memset(o, 0, n * sizeof(double));
    if (!check_init()) return;
    Builder bd;
    const int a = bd.add_shell(A), b = bd.add_shell(B);
    const int g = bd.add_grpp(UL, n_arep, arep, n_so, so, n_oc, ocp, ocs);
    const int c = bd.add_centre(C, g);
    bd.add_task(a, b, c);
    std::vector<double> out[4];
    if (run(bd, raw_so, out) != 0) return;
    for (int k = 0; k < 4; k++)
        if (outs[k]) memcpy(outs[k], out[k].data(), n * sizeof(double));
}

void libgrpp_type1_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *pot, double *matrix)
{
    one_task(A, B, C, pot, 0, nullptr, 0, nullptr, 0, nullptr, nullptr, 0, matrix, nullptr, nullptr, nullptr);
}

void libgrpp_type2_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *pot, double *matrix)
{
    one_task(A, B, C, nullptr, 1, &pot, 0, nullptr, 0, nullptr, nullptr, 0, matrix, nullptr, nullptr, nullptr);
}

void libgrpp_spin_orbit_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *pot,
                                  double *sx, double *sy, double *sz)
{
    one_task(A, B, C, nullptr, 0, nullptr, 1, &pot, 0, nullptr, nullptr, 1, nullptr, sx, sy, sz);
}

void libgrpp_outercore_potential_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, int noc,
                                           libgrpp_potential_t **pots, libgrpp_shell_t **ocs, double *arep,
                                           double *sx, double *sy, double *sz)
{
    one_task(A, B, C, nullptr, 0, nullptr, 0, nullptr, noc, pots, ocs, 0, arep, sx, sy, sz);
}

void libgrpp_full_grpp_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, libgrpp_grpp_t *g, double *C, double *arep,
                                 double *sx, double *sy, double *sz)
{
    one_task(A, B, C, g->U_L, g->n_arep, g->U_arep, g->n_esop, g->U_esop, g->n_oc_shells, g->U_oc, g->oc_shells, 0, arep,
             sx, sy, sz);
}

// ============================================================ gradients (grpp_integrals_gradient.c:123-393)
void libgrpp_full_grpp_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, libgrpp_grpp_t *g, double *C,
                                          double *D, double **ga, double **gx, double **gy, double **gz)
{
    gradient_impl(
        A, B, C, D,
        [&](Builder &bd) {
            return bd.add_grpp(g->U_L, g->n_arep, g->U_arep, g->n_esop, g->U_esop, g->n_oc_shells, g->U_oc, g->oc_shells);
        },
        0, ga, gx, gy, gz);
}

void libgrpp_type1_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *p,
                                      double *D, double **ga)
{
    gradient_impl(
        A, B, C, D, [&](Builder &bd) { return bd.add_grpp(p, 0, nullptr, 0, nullptr, 0, nullptr, nullptr); }, 0, ga,
        nullptr, nullptr, nullptr);
}

void libgrpp_type2_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *p,
                                      double *D, double **ga)
{
    gradient_impl(
        A, B, C, D, [&](Builder &bd) { return bd.add_grpp(nullptr, 1, &p, 0, nullptr, 0, nullptr, nullptr); }, 0, ga,
        nullptr, nullptr, nullptr);
}

// the reference scales the full-GRPP result back by (2L+1)/2 (grpp_integrals_gradient.c:229-237);
// here the spin-orbit blocks are produced without the factor in the first place
void libgrpp_spin_orbit_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, libgrpp_potential_t *p,
                                           double *D, double **gx, double **gy, double **gz)
{
    gradient_impl(
        A, B, C, D, [&](Builder &bd) { return bd.add_grpp(nullptr, 0, nullptr, 1, &p, 0, nullptr, nullptr); }, 1,
        nullptr, gx, gy, gz);
}

void libgrpp_outercore_potential_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, int noc,
                                                    libgrpp_potential_t **pots, libgrpp_shell_t **ocs, double *D,
                                                    double **ga, double **gx, double **gy, double **gz)
{
    gradient_impl(
        A, B, C, D, [&](Builder &bd) { return bd.add_grpp(nullptr, 0, nullptr, 0, nullptr, noc, pots, ocs); }, 0, ga,
        gx, gy, gz);
}

// ============================================================ batched API (libgrpp_b200.h)
int libgrpp_b200_last_error(void) { return grpp::last_error(); }
const char *libgrpp_b200_last_error_message(void) { return grpp::last_error_message(); }

int64_t libgrpp_b200_batch_output_size(const libgrpp_b200_batch_t *b) { return grpp::batch_output_size(b); }

int libgrpp_b200_full_grpp_batch(const libgrpp_b200_batch_t *b, int radial_mode, double *arep, double *sx, double *sy,
                                 double *sz)
{
    if (!check_init()) return LIBGRPP_B200_ERR_NOT_INIT;
    grpp::RunOptions opt;
    opt.radial_mode = radial_mode;
    return grpp::run_full_batch(b, opt, arep, sx, sy, sz);
}

int libgrpp_b200_set_device(int device) { return grpp::set_device(device); }

void *libgrpp_b200_host_alloc(size_t bytes) { return grpp::host_alloc(bytes); }

void libgrpp_b200_host_free(void *p) { grpp::host_free(p); }

int libgrpp_b200_fp64_peak(double *tflops) { return grpp::measure_fp64_peak(tflops); }

libgrpp_b200_plan_t *libgrpp_b200_plan_create(const libgrpp_b200_batch_t *b, int radial_mode)
{
    if (!check_init()) return nullptr;
    grpp::RunOptions opt;
    opt.radial_mode = radial_mode;
    return (libgrpp_b200_plan_t *)grpp::plan_create(b, opt);
}

libgrpp_b200_plan_t *libgrpp_b200_plan_create_ex(const libgrpp_b200_batch_t *b, int radial_mode, int assembly_threads)
{
    if (!check_init()) return nullptr;
    grpp::RunOptions opt;
    opt.radial_mode = radial_mode;
    opt.fin_nt = assembly_threads;
    return (libgrpp_b200_plan_t *)grpp::plan_create(b, opt);
}

int libgrpp_b200_autotune_assembly(const libgrpp_b200_batch_t *b, int radial_mode, double *rows, int cap)
{
    if (!check_init()) return LIBGRPP_B200_ERR_NOT_INIT;
    std::vector<std::array<double, 6>> r;
    const int rc = grpp::autotune_assembly(b, radial_mode, r);
    if (rc) return rc;
    for (int i = 0; i < (int)r.size() && i < cap; i++)
        for (int k = 0; k < 6; k++) rows[6 * i + k] = r[i][k];
    return (int)r.size();
}

void libgrpp_b200_autotune_reset(void) { grpp::autotune_reset(); }

int libgrpp_b200_plan_execute(libgrpp_b200_plan_t *plan)
{
    if (!plan) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, "null plan");
        return LIBGRPP_B200_ERR_INVALID;
    }
    return grpp::plan_run((grpp::Plan *)plan);
}

int libgrpp_b200_plan_outputs(libgrpp_b200_plan_t *plan, double *arep, double *sx, double *sy, double *sz)
{
    if (!plan) return LIBGRPP_B200_ERR_INVALID;
    return grpp::plan_outputs((grpp::Plan *)plan, arep, sx, sy, sz);
}

int libgrpp_b200_plan_stats(const libgrpp_b200_plan_t *plan, double *ms, int64_t *counts)
{
    if (!plan) return LIBGRPP_B200_ERR_INVALID;
    const grpp::RunStats *st = grpp::plan_stats((const grpp::Plan *)plan);
    if (ms) {
        ms[0] = st->ms_total;
        ms[1] = st->ms_mmd;
        ms[2] = st->ms_radial;
        ms[3] = st->ms_final;
        ms[4] = st->ms_screen;
    }
    if (counts) {
        counts[0] = st->n_tasks;
        counts[1] = st->n_radial;
        counts[2] = st->n_mmd;
        counts[3] = st->n_entries;
        counts[4] = grpp::plan_h2d_bytes((const grpp::Plan *)plan);
    }
    return 0;
}

int libgrpp_b200_plan_counters(const libgrpp_b200_plan_t *plan, uint64_t *counters, int n)
{
    if (!plan || n < 0 || n > 16) return LIBGRPP_B200_ERR_INVALID;
    const grpp::RunStats *st = grpp::plan_stats((const grpp::Plan *)plan);
    for (int i = 0; i < n; i++) counters[i] = st->radial_counters[i];
    return 0;
}

void libgrpp_b200_plan_destroy(libgrpp_b200_plan_t *plan) { grpp::plan_destroy((grpp::Plan *)plan); }

int libgrpp_b200_plan_set_counting(libgrpp_b200_plan_t *plan, int on)
{
    if (!plan) return LIBGRPP_B200_ERR_INVALID;
    grpp::plan_set_counting((grpp::Plan *)plan, on != 0);
    return 0;
}

static int grad_contract_impl(const libgrpp_b200_batch_t *b, int radial_mode, const int *shell_atom,
                              const int *centre_atom, const double *atom_xyz, int n_atoms, const int *bf_off, int n_bf,
                              const double *D, double *g, const double *task_weight, bool arep_only);

int libgrpp_b200_grpp_gradient_contract(const libgrpp_b200_batch_t *b, int radial_mode, const int *shell_atom,
                                        const int *centre_atom, const double *atom_xyz, int n_atoms, const int *bf_off,
                                        int n_bf, const double *D, double *g)
{
    return grad_contract_impl(b, radial_mode, shell_atom, centre_atom, atom_xyz, n_atoms, bf_off, n_bf, D, g, nullptr,
                              false);
}

// Symmetric density: the task (B, A, C) contributes to the arep gradient exactly what (A, B, C)
// does (D_BA = D_AB^T, V_BA = V_AB^T), and every spin-orbit contraction vanishes (the SO
// matrices and their derivatives are antisymmetric). The ordered task list is folded onto
// A <= B with weight 2 for A < B when both orders are present, spin-orbit potentials are left
// out of the derivative batch, and the spin-orbit gradient is returned as exact zeros.
int libgrpp_b200_grpp_gradient_contract_symmetric(const libgrpp_b200_batch_t *b, int radial_mode, const int *shell_atom,
                                                  const int *centre_atom, const double *atom_xyz, int n_atoms,
                                                  const int *bf_off, int n_bf, const double *D, double *g)
{
    if (!check_init()) return LIBGRPP_B200_ERR_NOT_INIT;
    grpp::set_error(0, "");
    auto invalid = [](const char *m) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, m);
        return LIBGRPP_B200_ERR_INVALID;
    };
    if (!b || !D || !g || n_bf <= 0 || b->n_tasks < 0) return invalid("gradient contraction: null argument or empty size");
    double dmax = 0.0;
    for (int64_t i = 0; i < (int64_t)n_bf * n_bf; i++) dmax = std::max(dmax, std::fabs(D[i]));
    for (int i = 0; i < n_bf; i++)
        for (int j = 0; j < i; j++)
            if (std::fabs(D[(int64_t)i * n_bf + j] - D[(int64_t)j * n_bf + i]) > 1e-14 * dmax)
                return invalid("gradient contraction: the density matrix is not symmetric");
    // fold (a, b, c) and (b, a, c) onto a <= b
    std::map<std::tuple<int, int, int>, int> seen;
    std::vector<int> fa, fb, fc;
    std::vector<double> w;
    for (int64_t t = 0; t < b->n_tasks; t++) {
        const int a = std::min(b->task_a[t], b->task_b[t]), bb = std::max(b->task_a[t], b->task_b[t]), c = b->task_c[t];
        auto it = seen.find({a, bb, c});
        if (it == seen.end()) {
            seen[{a, bb, c}] = (int)fa.size();
            fa.push_back(a);
            fb.push_back(bb);
            fc.push_back(c);
            w.push_back(1.0);
        } else {
            w[it->second] += 1.0;
        }
    }
    libgrpp_b200_batch_t v = *b;
    v.n_tasks = (int64_t)fa.size();
    v.task_a = fa.data();
    v.task_b = fb.data();
    v.task_c = fc.data();
    std::vector<int> no_so(b->n_grpps, 0);
    v.grpp_n_so = no_so.data();
    return grad_contract_impl(&v, radial_mode, shell_atom, centre_atom, atom_xyz, n_atoms, bf_off, n_bf, D, g, w.data(),
                              true);
}

static int grad_contract_impl(const libgrpp_b200_batch_t *b, int radial_mode, const int *shell_atom,
                              const int *centre_atom, const double *atom_xyz, int n_atoms, const int *bf_off, int n_bf,
                              const double *D, double *g, const double *task_weight, bool arep_only)
{
    if (!check_init()) return LIBGRPP_B200_ERR_NOT_INIT;
    grpp::set_error(0, "");
    auto invalid = [](const char *m) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, m);
        return LIBGRPP_B200_ERR_INVALID;
    };
    if (!b || !shell_atom || !centre_atom || !atom_xyz || !bf_off || !D || !g || n_atoms <= 0 || n_bf <= 0)
        return invalid("gradient contraction: null argument or empty size");
    const int ns = b->n_shells;
    const int kGL = grpp::kGradMaxL, Lmax_grad = kGL - 1;  // the L+1 shell must stay within the engine's limit
    // one component order per L: the batch's own lists (must agree within an L), else the generator
    std::vector<std::vector<int>> lists(kGL + 1);
    for (int s = 0; s < ns; s++) {
        const int L = b->shell_L[s];
        if (L < 0 || L > kGL) return invalid("gradient contraction: shell angular momentum outside 0..10");
        std::vector<int> cl(b->cart_list + 3 * b->shell_cart_off[s], b->cart_list + 3 * b->shell_cart_off[s] + 3 * ncart_h(L));
        if (lists[L].empty()) lists[L] = cl;
        else if (lists[L] != cl) return invalid("gradient contraction: shells of one L use different Cartesian orders");
    }
    for (int L = 0; L <= kGL; L++)
        if (lists[L].empty()) {
            lists[L].resize(3 * ncart_h(L));
            libgrpp_params.cartesian_generator(L, lists[L].data());
        }
    auto find = [&](int L, int x, int y, int z) {
        for (int i = 0; i < ncart_h(L); i++)
            if (lists[L][3 * i] == x && lists[L][3 * i + 1] == y && lists[L][3 * i + 2] == z) return i;
        return -1;
    };
    std::vector<int> tab((size_t)(kGL + 1) * grpp::kGradTabCart * 9, 0);
    for (int L = 0; L < kGL; L++)
        for (int i = 0; i < ncart_h(L); i++)
            for (int k = 0; k < 3; k++) {
                int c[3] = {lists[L][3 * i], lists[L][3 * i + 1], lists[L][3 * i + 2]};
                int *e = tab.data() + ((L * grpp::kGradTabCart + i) * 3 + k) * 3;
                e[0] = c[k];
                c[k] += 1;
                e[1] = find(L + 1, c[0], c[1], c[2]);
                c[k] -= 2;
                e[2] = c[k] >= 0 && L > 0 ? find(L - 1, c[0], c[1], c[2]) : -1;
            }
    // differentiated shells (diff_gaussian.c:35-63): L+1 with 2a N_L/N_{L+1}, L-1 with N_L/N_{L-1}
    std::vector<int> sL(b->shell_L, b->shell_L + ns), snp(b->shell_nprim, b->shell_nprim + ns),
        spo(b->shell_prim_off, b->shell_prim_off + ns), sco(b->shell_cart_off, b->shell_cart_off + ns);
    int nprim_tot = 0, ncart_tot = 0;
    for (int s = 0; s < ns; s++) {
        nprim_tot = std::max(nprim_tot, spo[s] + snp[s]);
        ncart_tot = std::max(ncart_tot, sco[s] + ncart_h(sL[s]));
    }
    std::vector<double> pc(b->prim_coef, b->prim_coef + nprim_tot), pa(b->prim_alpha, b->prim_alpha + nprim_tot),
        so(b->shell_origin, b->shell_origin + 3 * ns);
    std::vector<int> cart(b->cart_list, b->cart_list + 3 * ncart_tot);
    std::vector<int> up(ns, -1), dn(ns, -1);
    std::vector<uint8_t> used(ns, 0);
    for (int64_t t = 0; t < b->n_tasks; t++) {
        const int a = b->task_a[t], bb = b->task_b[t], c = b->task_c[t];
        if (a < 0 || a >= ns || bb < 0 || bb >= ns || c < 0 || c >= b->n_centres) return invalid("task index out of range");
        if (sL[a] > Lmax_grad || sL[bb] > Lmax_grad) return invalid("gradient contraction: shell L must be <= 9");
        if (shell_atom[a] < 0 || shell_atom[a] >= n_atoms || shell_atom[bb] < 0 || shell_atom[bb] >= n_atoms ||
            centre_atom[c] < 0 || centre_atom[c] >= n_atoms)
            return invalid("gradient contraction: atom index out of range");
        if (bf_off[a] < 0 || bf_off[a] + ncart_h(sL[a]) > n_bf || bf_off[bb] < 0 || bf_off[bb] + ncart_h(sL[bb]) > n_bf)
            return invalid("gradient contraction: basis offset outside the density matrix");
        used[a] = used[bb] = 1;
    }
    auto add_shell = [&](int s, int L, bool raise) {
        const int idx = (int)sL.size();
        sL.push_back(L);
        snp.push_back(snp[s]);
        spo.push_back((int)pc.size());
        sco.push_back((int)cart.size() / 3);
        for (int q = 0; q < 3 * ncart_h(L); q++) cart.push_back(lists[L][q]);
        for (int i = 0; i < snp[s]; i++) {
            const double al = pa[spo[s] + i];
            const double f = raise ? 2.0 * al * gaussian_norm(sL[s], al) / gaussian_norm(L, al)
                                   : gaussian_norm(sL[s], al) / gaussian_norm(L, al);
            pc.push_back(pc[spo[s] + i] * f);
            pa.push_back(al);
        }
        for (int d = 0; d < 3; d++) so.push_back(so[3 * s + d]);
        return idx;
    };
    for (int s = 0; s < ns; s++)
        if (used[s]) {
            up[s] = add_shell(s, sL[s] + 1, true);
            if (sL[s] > 0) dn[s] = add_shell(s, sL[s] - 1, false);
        }
    libgrpp_b200_batch_t sub = *b;
    sub.n_shells = (int)sL.size();
    sub.shell_L = sL.data();
    sub.shell_nprim = snp.data();
    sub.shell_prim_off = spo.data();
    sub.prim_coef = pc.data();
    sub.prim_alpha = pa.data();
    sub.shell_origin = so.data();
    sub.shell_cart_off = sco.data();
    sub.cart_list = cart.data();
    grpp::RunOptions opt;
    opt.radial_mode = radial_mode;
    const int64_t chunk = 16384;
    std::vector<int> ta, tb, tc;
    std::vector<grpp::GradTaskHost> gt;
    std::vector<double> out24;
    for (int64_t t0 = 0; t0 < b->n_tasks; t0 += chunk) {
        const int64_t t1 = std::min<int64_t>(b->n_tasks, t0 + chunk);
        ta.clear();
        tb.clear();
        tc.clear();
        gt.clear();
        auto add = [&](int x, int y, int c) {
            ta.push_back(x);
            tb.push_back(y);
            tc.push_back(c);
            return (int)ta.size() - 1;
        };
        for (int64_t t = t0; t < t1; t++) {
            const int a = b->task_a[t], bb = b->task_b[t], c = b->task_c[t];
            grpp::GradTaskHost h;
            h.t_ad = dn[a] >= 0 ? add(dn[a], bb, c) : -1;
            h.t_au = add(up[a], bb, c);
            h.t_bd = dn[bb] >= 0 ? add(a, dn[bb], c) : -1;
            h.t_bu = add(a, up[bb], c);
            h.la = sL[a];
            h.lb = sL[bb];
            h.d_row = bf_off[a];
            h.d_col = bf_off[bb];
            gt.push_back(h);
        }
        sub.n_tasks = (int64_t)ta.size();
        sub.task_a = ta.data();
        sub.task_b = tb.data();
        sub.task_c = tc.data();
        out24.assign((size_t)(t1 - t0) * 24, 0.0);
        const int rc = grpp::run_grad_contract(&sub, opt, gt.data(), t1 - t0, tab.data(), D, n_bf, out24.data());
        if (rc) return rc;
        // which atoms receive which side, with which sign (grpp_integrals_gradient.c:280-393)
        for (int64_t t = t0; t < t1; t++) {
            const int a = b->task_a[t], bb = b->task_b[t], c = b->task_c[t];
            const double *A = b->shell_origin + 3 * a, *B = b->shell_origin + 3 * bb, *C = b->centre_origin + 3 * c;
            const int atoms[3] = {shell_atom[a], shell_atom[bb], centre_atom[c]};
            const double *o = out24.data() + (t - t0) * 24;
            const double wt = task_weight ? task_weight[t] : 1.0;
            const int nm = arep_only ? 1 : 4;
            for (int q = 0; q < 3; q++) {
                const int at = atoms[q];
                if ((q > 0 && atoms[0] == at) || (q > 1 && atoms[1] == at)) continue;
                for (const GradContribution &tcn : gradient_terms(A, B, C, atom_xyz + 3 * at)) {
                    const int side = tcn.diff_bra ? 0 : 1;
                    for (int k = 0; k < 3; k++)
                        for (int m = 0; m < nm; m++)
                            g[((size_t)m * n_atoms + at) * 3 + k] += wt * (tcn.factor * o[side * 12 + k * 4 + m]);
                }
            }
        }
    }
    return 0;
}

int libgrpp_b200_plan_learned_stats(const libgrpp_b200_plan_t *plan, double *ms_predict, int64_t *fallbacks)
{
    if (!plan) return LIBGRPP_B200_ERR_INVALID;
    const grpp::RunStats *st = grpp::plan_stats((const grpp::Plan *)plan);
    if (ms_predict) *ms_predict = st->ms_predict;
    if (fallbacks) *fallbacks = st->fallbacks;
    return 0;
}

int libgrpp_b200_set_level_model(const float *params)
{
    if (!params) return LIBGRPP_B200_ERR_INVALID;
    return grpp::set_level_model(params);
}

int libgrpp_b200_level_samples(const libgrpp_b200_batch_t *b, float *features, int8_t *levels, int64_t *n_items)
{
    if (!check_init()) return LIBGRPP_B200_ERR_NOT_INIT;
    if (!b || !features || !levels || !n_items) return LIBGRPP_B200_ERR_INVALID;
    return grpp::level_samples(b, features, levels, n_items);
}

int libgrpp_b200_mlp_grad(const float *params, const float *features, const int8_t *levels, int n, float *grad,
                          float *loss)
{
    if (!params || !features || !levels || !grad || !loss) return LIBGRPP_B200_ERR_INVALID;
    return grpp::mlp_grad(params, features, levels, n, grad, loss);
}

int libgrpp_b200_mlp_train(const float *features, const int8_t *levels, int64_t n, int epochs, int batch, float lr,
                           uint32_t seed, float *params, float *epoch_loss)
{
    if (!params || !features || !levels) return LIBGRPP_B200_ERR_INVALID;
    return grpp::mlp_train(features, levels, n, epochs, batch, lr, seed, params, epoch_loss);
}

int libgrpp_b200_mlp_predict(const float *params, const float *features, int64_t n, int8_t *levels)
{
    if (!params || !features || !levels) return LIBGRPP_B200_ERR_INVALID;
    return grpp::mlp_predict(params, features, n, levels);
}

}  // extern "C"
// ============================================================ one-electron integrals
// libgrpp/overlap.c, kinetic.c, momentum.c, overlap_gradient.c, nuclear_attraction.c,
// nuclear_models.c: the same entry points, evaluated on the GPU (batches of one).

void libgrpp_overlap_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *matrix)
{
    onee_single(A, B, 0, matrix, nullptr, nullptr);
}

void libgrpp_kinetic_energy_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *matrix)
{
    onee_single(A, B, 1, matrix, nullptr, nullptr);
}

void libgrpp_momentum_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *mx, double *my, double *mz)
{
    onee_single(A, B, 2, mx, my, mz);
}

// overlap_gradient.c:27-141: d<A|B>/dA = +<dA|B>, d<A|B>/dB = -<dA|B>, zero for A = B
void libgrpp_overlap_integrals_gradient(libgrpp_shell_t *A, libgrpp_shell_t *B, double *D, double **grad)
{
    const int nA = A->cart_size, nB = B->cart_size, n = nA * nB;
    for (int k = 0; k < 3; k++) memset(grad[k], 0, n * sizeof(double));
    if (!check_init() || points_equal(A->origin, B->origin)) return;
    double factors[2];
    int nf = 0;
    if (points_equal(A->origin, D)) factors[nf++] = +1.0;
    if (points_equal(B->origin, D)) factors[nf++] = -1.0;
    if (nf == 0) return;
    libgrpp_shell_t *Ad = shell_down(A), *Au = shell_up(A);
    std::vector<double> down(Ad ? Ad->cart_size * nB : 1), up(Au->cart_size * nB);
    if (Ad) onee_single(Ad, B, 0, down.data(), nullptr, nullptr);
    onee_single(Au, B, 0, up.data(), nullptr, nullptr);
    for (int f = 0; f < nf; f++)
        for (int k = 0; k < 3; k++)
            for (int i = 0; i < nA; i++)
                for (int j = 0; j < nB; j++) {
                    int bra[3] = {A->cart_list[3 * i], A->cart_list[3 * i + 1], A->cart_list[3 * i + 2]};
                    const int *ket = B->cart_list + 3 * j;
                    const int idx = i * nB + j;
                    // the L-1 term only where the exponent is positive: libgrpp also forms it for a zero
                    // exponent, reading past its L-1 block and multiplying by 0
                    if (Ad && bra[k] > 0) {
                        bra[k] -= 1;
                        const int bi = nlm_to_linear(bra), ki = nlm_to_linear(ket);
                        bra[k] += 1;
                        grad[k][idx] -= factors[f] * bra[k] * down[nB * bi + ki];
                    }
                    bra[k] += 1;
                    const int bi = nlm_to_linear(bra), ki = nlm_to_linear(ket);
                    bra[k] -= 1;
                    grad[k][idx] += factors[f] * up[nB * bi + ki];
                }
    if (Ad) libgrpp_delete_shell(Ad);
    libgrpp_delete_shell(Au);
}

void libgrpp_nuclear_attraction_integrals(libgrpp_shell_t *A, libgrpp_shell_t *B, double *charge_origin, int charge,
                                          int nuclear_model, double *model_params, double *coulomb_matrix)
{
    const int n = A->cart_size * B->cart_size;
    memset(coulomb_matrix, 0, n * sizeof(double));
    if (!check_init()) return;
    Builder bd;
    const int ia = bd.add_shell(A), ib = bd.add_shell(B);
    bd.add_centre(charge_origin, 0);
    bd.add_task(ia, ib, 0);
    bd.grpp_UL.push_back(-1);  // one empty GRPP: the centre needs an operator index only
    bd.grpp_arep_off.push_back(0);
    bd.grpp_n_arep.push_back(0);
    bd.grpp_so_off.push_back(0);
    bd.grpp_n_so.push_back(0);
    bd.grpp_oc_off.push_back(0);
    bd.grpp_n_oc.push_back(0);
    libgrpp_b200_batch_t v = bd.view();
    const double z = charge;
    double prm[3] = {0, 0, 0};
    const int np = nuclear_model == LIBGRPP_NUCLEAR_MODEL_FERMI ? 2 : (nuclear_model == LIBGRPP_NUCLEAR_MODEL_FERMI_BUBBLE ? 3 : 1);
    if (nuclear_model != LIBGRPP_NUCLEAR_MODEL_POINT_CHARGE && nuclear_model != LIBGRPP_NUCLEAR_MODEL_POINT_CHARGE_NUMERICAL) {
        if (!model_params) {
            grpp::set_error(LIBGRPP_B200_ERR_INVALID, "nuclear model parameters missing");
            return;
        }
        for (int q = 0; q < np; q++) prm[q] = model_params[q];
    }
    libgrpp_b200_nuclear_attraction_batch(&v, nuclear_model, &z, prm, coulomb_matrix);
}

void libgrpp_nuclear_attraction_integrals_point_charge(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, int charge,
                                                       double *m)
{
    libgrpp_nuclear_attraction_integrals(A, B, C, charge, LIBGRPP_NUCLEAR_MODEL_POINT_CHARGE, nullptr, m);
}
// The model-specific wrappers pass libgrpp_nuclear_attraction_integrals the array
// {charge, model parameters...}, which the generic function reads from its first element on
// (nuclear_attraction.c:125-170, 193-236): in libgrpp these wrappers therefore evaluate the
// model with the charge as its first parameter (R_rms, or c) and the remaining parameters
// shifted by one. The same array is passed here, so the wrappers return libgrpp's values;
// libgrpp_nuclear_attraction_integrals with model_params = {R_rms} / {c, a} / {c, a, k} is the
// form that evaluates the model with the given parameters.
void libgrpp_nuclear_attraction_integrals_charged_ball(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, int charge,
                                                       double r_rms, double *m)
{
    double p[10] = {(double)charge, r_rms};
    libgrpp_nuclear_attraction_integrals(A, B, C, charge, LIBGRPP_NUCLEAR_MODEL_CHARGED_BALL, p, m);
}
void libgrpp_nuclear_attraction_integrals_gaussian_model(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, int charge,
                                                         double r_rms, double *m)
{
    double p[10] = {(double)charge, r_rms};
    libgrpp_nuclear_attraction_integrals(A, B, C, charge, LIBGRPP_NUCLEAR_MODEL_GAUSSIAN, p, m);
}
void libgrpp_nuclear_attraction_integrals_fermi_model(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, int charge,
                                                      double fermi_param_c, double fermi_param_a, double *m)
{
    double p[10] = {(double)charge, fermi_param_c, fermi_param_a};
    libgrpp_nuclear_attraction_integrals(A, B, C, charge, LIBGRPP_NUCLEAR_MODEL_FERMI, p, m);
}
void libgrpp_nuclear_attraction_integrals_fermi_bubble_model(libgrpp_shell_t *A, libgrpp_shell_t *B, double *C, int charge,
                                                             double param_c, double param_a, double param_k, double *m)
{
    double p[10] = {(double)charge, param_c, param_a, param_k};
    libgrpp_nuclear_attraction_integrals(A, B, C, charge, LIBGRPP_NUCLEAR_MODEL_FERMI_BUBBLE, p, m);
}

// ---- nuclear charge models (nuclear_models.c): host functions
double libgrpp_estimate_nuclear_rms_radius_johnson_1985(int A) { return 0.836 * pow(A, 1.0 / 3.0) + 0.570; }
double libgrpp_estimate_nuclear_rms_radius_golovko_2008(int A) { return 0.77 * pow(A, 1.0 / 3.0) + 0.98; }
int libgrpp_estimate_fermi_model_parameters(double R_rms, double *c, double *a)
{
    const double t = 2.3;
    *a = t / (4 * log(3));
    const double c2 = 5.0 / 3.0 * R_rms * R_rms - 7.0 / 3.0 * M_PI * M_PI * (*a) * (*a);
    if (c2 < 0) return -1;
    *c = sqrt(c2);
    return 1;
}
double libgrpp_charge_density_ball(double r, double Z, double R_rms)
{
    const double R0 = sqrt(5.0 / 3.0) * R_rms;
    return r <= R0 ? 3.0 * Z / (4.0 * M_PI * R0 * R0 * R0) : 0.0;
}
double libgrpp_charge_density_gaussian(double r, double Z, double R_rms)
{
    const double xi = 3.0 / (2.0 * R_rms * R_rms);
    return Z * pow(xi / M_PI, 1.5) * exp(-xi * r * r);
}
double libgrpp_charge_density_fermi(double r, double Z, double c, double a)
{
    const double N = grpp::fermi_norm(c, a, grpp::fermi_table());
    return 3.0 * Z / (4 * M_PI * c * c * c * N) / (1.0 + exp((r - c) / a));
}
double libgrpp_charge_density_fermi_bubble(double r, double Z, double c, double a, double k)
{
    const double Nk = grpp::fermi_bubble_norm(c, a, k, grpp::fermi_table());
    return 3.0 * Z / (4 * M_PI * c * c * c * Nk) * (1 + k * pow(r / c, 2)) / (1.0 + exp((r - c) / a));
}
double libgrpp_rms_radius_fermi(int Z, double c, double a)
{
    const double *tab = grpp::fermi_table();
    const double N = grpp::fermi_norm(c, a, tab), rho0 = 3.0 * Z / (4 * M_PI * c * c * c * N);
    const double r2 = 4 * M_PI * rho0 / Z * pow(c, 5) / 5.0 *
                      (1.0 + 10.0 / 3.0 * a * a * M_PI * M_PI / (c * c) + 7.0 / 3.0 * pow(M_PI, 4) * pow(a, 4) / pow(c, 4) -
                       120.0 * pow(a, 5) / pow(c, 5) * grpp::fermi_sk(5, -c / a, tab));
    return sqrt(r2);
}
double libgrpp_rms_radius_fermi_bubble(int Z, double c, double a, double k)
{
    const double *tab = grpp::fermi_table();
    const double Nk = grpp::fermi_bubble_norm(c, a, k, tab), rho0 = 3.0 * Z / (4 * M_PI * c * c * c * Nk);
    const double part_r4 = pow(c, 5) / 5.0 *
                           (1.0 + 10.0 / 3.0 * a * a * M_PI * M_PI / (c * c) + 7.0 / 3.0 * pow(M_PI, 4) * pow(a, 4) / pow(c, 4) -
                            120.0 * pow(a, 5) / pow(c, 5) * grpp::fermi_sk(5, -c / a, tab));
    const double part_r6 = pow(c, 7) / 7.0 *
                           (1.0 + 7.0 * a * a * M_PI * M_PI / (c * c) + 49.0 / 3.0 * pow(M_PI, 4) * pow(a, 4) / pow(c, 4) +
                            31.0 / 3.0 * pow(M_PI, 6) * pow(a, 6) / pow(c, 6) -
                            5040.0 * pow(a, 7) / pow(c, 7) * grpp::fermi_sk(7, -c / a, tab));
    return sqrt(4 * M_PI * rho0 / Z * (part_r4 + k / (c * c) * part_r6));
}
double libgrpp_coulomb_potential_point(double r, double Z) { return -Z / r; }
double libgrpp_coulomb_potential_ball(double r, double Z, double R_rms) { return grpp::coulomb_ball(r, Z, R_rms); }
double libgrpp_coulomb_potential_gaussian(double r, double Z, double R_rms) { return grpp::coulomb_gauss(r, Z, R_rms); }
double libgrpp_coulomb_potential_fermi(double r, double Z, double c, double a)
{
    return grpp::coulomb_fermi(r, Z, c, a, grpp::fermi_table());
}
double libgrpp_coulomb_potential_fermi_bubble(double r, double Z, double c, double a, double k)
{
    return grpp::coulomb_fermi_bubble(r, Z, c, a, k, grpp::fermi_table());
}

// ---- batched forms (no counterpart in libgrpp)
int libgrpp_b200_onee_batch(const libgrpp_b200_batch_t *batch, int kind, double *out0, double *out1, double *out2)
{
    if (!check_init()) return LIBGRPP_B200_ERR_NOT_INIT;
    if (!batch || !out0 || (kind == LIBGRPP_B200_ONEE_MOMENTUM && (!out1 || !out2))) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, "one-electron batch: null argument");
        return LIBGRPP_B200_ERR_INVALID;
    }
    return grpp::run_onee_batch(batch, kind, out0, out1, out2);
}

int libgrpp_b200_nuclear_attraction_batch(const libgrpp_b200_batch_t *batch, int nuclear_model, const double *centre_charge,
                                          const double *centre_params, double *out)
{
    if (!check_init()) return LIBGRPP_B200_ERR_NOT_INIT;
    auto invalid = [](const char *m) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, m);
        return LIBGRPP_B200_ERR_INVALID;
    };
    if (!batch || !centre_charge || !out) return invalid("nuclear attraction batch: null argument");
    if (batch->n_tasks == 0) return 0;
    const int nc = batch->n_centres;
    if (nc <= 0) return invalid("nuclear attraction batch: no centres");
    if (nuclear_model == LIBGRPP_NUCLEAR_MODEL_POINT_CHARGE) {
        // libgrpp evaluates the point charge through its type 1 McMurchie-Davidson code with a zero
        // exponent (nuclear_attraction.c:106-117): here every centre gets a GRPP whose U_L is
        // -Z r^(1-2) exp(0 r^2), and the batch runs through the GRPP engine
        std::vector<int> pL(nc, 0), pJ(nc, 0), pn(nc, 1), po(nc), pw(nc, 1), g(nc), z0(nc, 0), cg(nc);
        std::vector<double> pc(nc), pa(nc, 0.0);
        for (int c = 0; c < nc; c++) {
            po[c] = c;
            pc[c] = -centre_charge[c];
            g[c] = c;
            cg[c] = c;
        }
        libgrpp_b200_batch_t v = *batch;
        v.n_pots = nc;
        v.pot_L = pL.data();
        v.pot_J = pJ.data();
        v.pot_nprim = pn.data();
        v.pot_prim_off = po.data();
        v.pot_powers = pw.data();
        v.pot_coef = pc.data();
        v.pot_alpha = pa.data();
        v.n_grpps = nc;
        v.grpp_UL = g.data();
        v.grpp_arep_off = z0.data();
        v.grpp_n_arep = z0.data();
        v.grpp_so_off = z0.data();
        v.grpp_n_so = z0.data();
        v.grpp_oc_off = z0.data();
        v.grpp_n_oc = z0.data();
        v.grpp_pot_list = z0.data();
        v.grpp_oc_pot = z0.data();
        v.grpp_oc_shell = z0.data();
        v.centre_grpp = cg.data();
        const int64_t n = grpp::batch_output_size(&v);
        std::vector<double> so[3];
        for (auto &x : so) x.assign(std::max<int64_t>(n, 1), 0.0);
        grpp::RunOptions opt;
        return grpp::run_full_batch(&v, opt, out, so[0].data(), so[1].data(), so[2].data());
    }
    int model;
    switch (nuclear_model) {
    case LIBGRPP_NUCLEAR_MODEL_POINT_CHARGE_NUMERICAL: model = grpp::kPotPointNum; break;
    case LIBGRPP_NUCLEAR_MODEL_CHARGED_BALL: model = grpp::kPotBall; break;
    case LIBGRPP_NUCLEAR_MODEL_GAUSSIAN: model = grpp::kPotGauss; break;
    case LIBGRPP_NUCLEAR_MODEL_FERMI: model = grpp::kPotFermi; break;
    case LIBGRPP_NUCLEAR_MODEL_FERMI_BUBBLE: model = grpp::kPotFermiBubble; break;
    default: return invalid("unknown nuclear charge distribution model");
    }
    if (model != grpp::kPotPointNum && !centre_params) return invalid("nuclear model parameters missing");
    std::vector<double> prm((size_t)4 * nc, 0.0);
    for (int c = 0; c < nc; c++) {
        prm[4 * c] = centre_charge[c];
        if (model != grpp::kPotPointNum)
            for (int q = 0; q < 3; q++) prm[4 * c + 1 + q] = centre_params[3 * c + q];
    }
    // nuclear_attraction.c:50-54: primitive pairs with |c_i c_j| < 1e-13 are skipped
    return grpp::run_type1_numeric_batch(batch, model, prm.data(), libgrpp_params.radial_tolerance, 1e-13, out);
}

int libgrpp_b200_type1_numeric_batch(const libgrpp_b200_batch_t *batch, double *arep)
{
    if (!check_init()) return LIBGRPP_B200_ERR_NOT_INIT;
    if (!batch || !arep) {
        grpp::set_error(LIBGRPP_B200_ERR_INVALID, "numeric type 1 batch: null argument");
        return LIBGRPP_B200_ERR_INVALID;
    }
    return grpp::run_type1_numeric_batch(batch, grpp::kPotGrpp, nullptr, libgrpp_params.radial_tolerance, 0.0, arep);
}

#pragma GCC visibility pop
