// instance.cpp -- host tables of one hierarchy instance.
//
// Restates dm-heom/src/heom/instance.cpp:25-71 (table set-up) and
// precompute_baths_input (:155-273) in the same complex arithmetic and
// operation order, so that the double results round identically.
#include <cmath>

#include "heom_host.hpp"

namespace heomhost {

#include "pade_tables.inc"

heom_instance_desc instance::desc() const
{
    heom_instance_desc d{};
    d.states = sys.states;
    d.matsubaras = sys.matsubaras;
    d.baths = sys.baths;
    d.baths_per_state = sys.baths_per_state;
    d.ado_width = width;
    d.ado_depth = sys.depth;
    d.matrices = matrices;
    d.first_non_plus_id = first_non_plus;
    d.baths_coupling = sys.coupling.data();
    d.hamiltonian = hamiltonian.data();
    d.ado_tuples = tuples.data();
    d.ado_plus = plus.data();
    d.ado_minus = minus.data();
    d.pf_same_sum = pf_same_sum.data();
    d.pf_same = pf_same.data();
    d.pf_circ = pf_circ.data();
    d.cbk = cbk.data();
    d.cbk_sqrt = cbk_sqrt.data();
    return d;
}

void validate_system(const system_params& s)
{
    // config.cpp:117-174 (the checks that concern the derivative path)
    if (s.states <= 0) throw config_error("system.sites must be > 0");
    if (s.depth <= 0) throw config_error("system.ado_depth must be > 0");
    if ((int64_t)s.hamiltonian.size() != (int64_t)s.states * s.states)
        throw config_error("system.hamiltonien must be a system.sites by system.sites matrix");
    for (int i = 0; i < s.states; ++i)
        for (int j = 0; j < s.states; ++j) {
            const complex_t a = s.hamiltonian[i * s.states + j], b = s.hamiltonian[j * s.states + i];
            if (a != std::conj(b)) throw config_error("system.hamiltonien must be hermitian");
        }
    if (s.baths <= 0) throw config_error("baths.number must be > 0");
    if (s.baths_per_state <= 0) throw config_error("baths.max_per_site must be > 0");
    if (s.baths_per_state > s.baths) throw config_error("baths.max_per_site must be <= baths.number");
    if ((int64_t)s.coupling.size() != (int64_t)s.states * s.baths_per_state)
        throw config_error("baths.coupling must be a system.sites by baths_max_per_site_ matrix");
    for (int32_t c : s.coupling)
        if (!(c < s.baths))
            throw config_error("baths.coupling values must between 0 and baths.number, or negative for non-coupling");
    if ((int32_t)s.lambda.size() != s.baths) throw config_error("baths.lambda must have a length of baths.number");
    if ((int32_t)s.invnu.size() != s.baths) throw config_error("baths.invnu must have a length of baths.number");
    for (double v : s.invnu)
        if (!(v > 0)) throw config_error("baths.invnu must have values > 0");
    if ((int32_t)s.omega.size() != s.baths) throw config_error("baths.Omega must have a length of baths.number");
    if (s.matsubaras < 1 || s.matsubaras > max_pade)
        throw config_error("baths.matsubaras must be between 1 and 10 (Pade tables)");
    if (!(s.temperature > 0)) throw config_error("baths.temperature must be > 0");
}

system_params system_from_desc(const heom_system_desc& d)
{
    if (!d.hamiltonian || !d.baths_coupling || !d.lambda || !d.invnu || !d.omega)
        throw config_error("system description has a NULL array");
    system_params s;
    s.states = d.sites;
    s.depth = d.ado_depth;
    s.baths = d.baths;
    s.baths_per_state = d.baths_max_per_site;
    s.matsubaras = d.matsubaras;
    s.temperature = d.temperature;
    if (d.sites <= 0 || d.baths <= 0 || d.baths_max_per_site <= 0) throw config_error("sizes must be > 0");
    const int64_t nn = (int64_t)d.sites * d.sites;
    s.hamiltonian.resize(nn);
    for (int64_t q = 0; q < nn; ++q) // parser::matrix::scale (config.cpp:187)
        s.hamiltonian[q] = complex_t(d.hamiltonian[2 * q] * invcm_to_joule, d.hamiltonian[2 * q + 1] * invcm_to_joule);
    s.coupling.assign(d.baths_coupling, d.baths_coupling + (int64_t)d.sites * d.baths_max_per_site);
    for (int b = 0; b < d.baths; ++b) {
        s.lambda.push_back(d.lambda[b] * invcm_to_joule);            // :188
        s.omega.push_back(d.omega[b] * (invcm_to_joule / h_bar));    // :189
        s.invnu.push_back(d.invnu[b] * 1.0E-15);                     // :190
    }
    return s;
}

instance make_instance(const system_params& sys)
{
    validate_system(sys);
    instance in;
    in.sys = sys;
    hierarchy_graph g(sys.baths * sys.matsubaras, sys.depth);
    in.matrices = g.nodes();
    in.width = (int32_t)g.width();
    in.first_non_plus = g.first_non_plus_uid();
    in.tuples = g.tuples();
    in.plus = g.plus();
    in.minus = g.minus();
    const int N = sys.states;
    in.hamiltonian.resize(2 * N * N);
    for (int q = 0; q < N * N; ++q) {
        in.hamiltonian[2 * q] = sys.hamiltonian[q].real();
        in.hamiltonian[2 * q + 1] = sys.hamiltonian[q].imag();
    }

    // precompute_baths_input (instance.cpp:155-273)
    const int M = sys.matsubaras;
    const int B = sys.baths;
    const int row = (M - 1) * max_pade;
    const double hbar = h_bar;
    const double beta = 1.0 / (k_b * sys.temperature);
    in.pf_same.assign(2 * B, 0.0);
    in.pf_circ.assign(2 * B, 0.0);
    in.cbk.assign(2 * B * M, 0.0);
    in.cbk_sqrt.assign(B * M, 0.0);
    for (int b = 0; b < B; ++b) {
        const complex_t lambda_b{sys.lambda[b]};
        const complex_t nu_b{1.0 / sys.invnu[b], sys.omega[b]};
        const complex_t pfc = nu_b * lambda_b / hbar;                       // :176
        complex_t aux = 2.0 * lambda_b / (beta * hbar * hbar * nu_b);       // :177
        in.pf_circ[2 * b] = pfc.real();
        in.pf_circ[2 * b + 1] = pfc.imag();
        for (int k = 0; k < M; ++k) {
            complex_t cb, nubk;
            if (k == 0) {
                complex_t auxsum = 0.0;
                for (int j = 0; j < M; ++j) {
                    const double eta = (double)heom_eta_pade[row + j];
                    const double xi = (double)heom_xi_pade[row + j];
                    auxsum += (2.0 * eta * nu_b * nu_b) / (xi * xi / (beta * beta * hbar * hbar) - nu_b * nu_b);
                }
                cb = 2.0 * lambda_b / (beta * hbar) * (1.0 - auxsum);
                nubk = nu_b;
            } else {
                const double eta = (double)heom_eta_pade[row + k];
                const double xi = (double)heom_xi_pade[row + k];
                cb = 4.0 * lambda_b * nu_b / (beta * beta * hbar * hbar) * (eta * xi) /
                     (xi * xi / (beta * beta * hbar * hbar) - nu_b * nu_b);
                nubk = xi / (beta * hbar);
            }
            in.cbk[2 * (b * M + k)] = cb.real();
            in.cbk[2 * (b * M + k) + 1] = cb.imag();
            in.cbk_sqrt[b * M + k] = std::sqrt(std::abs(cb));
            aux -= cb / (hbar * nubk);
        }
        in.pf_same[2 * b] = aux.real();
        in.pf_same[2 * b + 1] = aux.imag();
    }
    const int64_t W = in.width;
    in.pf_same_sum.assign(2 * in.matrices, 0.0);
    for (int64_t id = 0; id < in.matrices; ++id) { // :227-262, long double sums
        long double zr = 0.0L, zi = 0.0L;
        for (int b = 0; b < B; ++b) {
            const complex_t nu_b{1.0 / sys.invnu[b], sys.omega[b]};
            for (int k = 0; k < M; ++k) {
                long double nr, ni;
                if (k == 0) {
                    nr = static_cast<long double>(nu_b.real());
                    ni = static_cast<long double>(nu_b.imag());
                } else {
                    nr = heom_xi_pade[row + k] / static_cast<long double>(beta * hbar);
                    ni = 0.0L;
                }
                const int m = b * M + k;
                zr -= nr * static_cast<long double>(in.tuples[id * W + m]);
                zi -= ni * static_cast<long double>(in.tuples[id * W + m]);
            }
        }
        in.pf_same_sum[2 * id] = (double)zr;
        in.pf_same_sum[2 * id + 1] = (double)zi;
    }
    return in;
}

// Derivatives of pf_same, pf_circ and cbk (the formulas of make_instance
// above, instance.cpp:155-221 of the reference) with respect to theta = 0:
// lambda of every bath moved together (per J), theta = 1: gamma = 1/invnu of
// every bath moved together (per 1/s).  With nu = gamma + i Omega and
// a = 1 / (beta hbar):
//   pf_circ = nu lambda / hbar
//   cb_0    = 2 lambda a (1 - S),  S = sum_j 2 eta_j nu^2 / (X_j - nu^2),  X_j = xi_j^2 a^2
//   cb_k    = 4 lambda nu a^2 eta_k xi_k / (X_k - nu^2)                     (k >= 1)
//   pf_same = 2 lambda a / (hbar nu) - cb_0 / (hbar nu) - sum_k cb_k / (hbar xi_k a)
// pf_same_sum = -sum n_{b,k} nu_{b,k} changes with gamma only (by -n_{b,0}).
bath_derivs bath_derivatives(const system_params& sys)
{
    const int M = sys.matsubaras, B = sys.baths;
    const int row = (M - 1) * max_pade;
    const double hbar = h_bar;
    const double beta = 1.0 / (k_b * sys.temperature);
    const double a = 1.0 / (beta * hbar);
    bath_derivs d;
    for (int th = 0; th < 2; ++th) {
        d.pf_same[th].assign(2 * B, 0.0);
        d.pf_circ[th].assign(2 * B, 0.0);
        d.cbk[th].assign(2 * B * M, 0.0);
    }
    auto put = [](std::vector<double>& v, int q, complex_t z) {
        v[2 * q] = z.real();
        v[2 * q + 1] = z.imag();
    };
    for (int b = 0; b < B; ++b) {
        const double lam = sys.lambda[b];
        const complex_t nu{1.0 / sys.invnu[b], sys.omega[b]};
        put(d.pf_circ[0], b, nu / hbar);
        put(d.pf_circ[1], b, complex_t(lam / hbar));
        complex_t dsame[2] = {2.0 * a / (hbar * nu), -2.0 * lam * a / (hbar * nu * nu)};
        for (int k = 0; k < M; ++k) {
            complex_t dcb[2];
            if (k == 0) {
                complex_t S = 0.0, dS = 0.0;
                for (int j = 0; j < M; ++j) {
                    const double eta = (double)heom_eta_pade[row + j];
                    const double xi = (double)heom_xi_pade[row + j];
                    const double X = xi * xi * a * a;
                    const complex_t den = X - nu * nu;
                    S += 2.0 * eta * nu * nu / den;
                    dS += 4.0 * eta * nu * X / (den * den);
                }
                const complex_t cb = 2.0 * lam * a * (1.0 - S);
                dcb[0] = 2.0 * a * (1.0 - S);
                dcb[1] = -2.0 * lam * a * dS;
                dsame[0] -= dcb[0] / (hbar * nu);
                dsame[1] -= dcb[1] / (hbar * nu) - cb / (hbar * nu * nu);
            } else {
                const double eta = (double)heom_eta_pade[row + k];
                const double xi = (double)heom_xi_pade[row + k];
                const double X = xi * xi * a * a;
                const complex_t den = X - nu * nu;
                dcb[0] = 4.0 * nu * a * a * eta * xi / den;
                dcb[1] = 4.0 * lam * a * a * eta * xi * (X + nu * nu) / (den * den);
                const double nuk = xi * a;
                dsame[0] -= dcb[0] / (hbar * nuk);
                dsame[1] -= dcb[1] / (hbar * nuk);
            }
            put(d.cbk[0], b * M + k, dcb[0]);
            put(d.cbk[1], b * M + k, dcb[1]);
        }
        put(d.pf_same[0], b, dsame[0]);
        put(d.pf_same[1], b, dsame[1]);
    }
    return d;
}

} // namespace heomhost
