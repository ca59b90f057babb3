// spectra.cpp -- state systems with a ground state and dipole matrices for
// the spectroscopy applications (linear absorption, circular dichroism).
//
// The sites -> states map follows dm-heom/src/heom/sites_to_states.cpp:16-28,
// 44-55, 131-142; the dipole matrices follow dipole_matrix.cpp:105-131 and
// dipole_matrix.hpp:30-75 for the pseudo pathway of
// dipole_pseudo_pathway.hpp:22-27.
#include <stdexcept>

#include "heom_host.hpp"

namespace heomhost {

system_params state_system(const system_params& sites, sites_to_states_mode mode)
{
    if (mode == sites_to_states_mode::identity) return sites;
    // with ground state: one more state (index 0) with a zero row and column
    // of H and no bath coupling
    system_params s = sites;
    const int n = sites.states, m = n + 1;
    s.states = m;
    s.hamiltonian.assign((size_t)m * m, complex_t(0.0, 0.0));
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) s.hamiltonian[(size_t)(i + 1) * m + (j + 1)] = sites.hamiltonian[(size_t)i * n + j];
    s.coupling.assign((size_t)m * sites.baths_per_state, -1);
    for (int i = 0; i < n; ++i)
        for (int b = 0; b < sites.baths_per_state; ++b)
            s.coupling[(size_t)(i + 1) * sites.baths_per_state + b] = sites.coupling[(size_t)i * sites.baths_per_state + b];
    return s;
}

std::vector<double> dipole_matrix(const std::vector<double>& v)
{
    const size_t m = v.size() + 1;
    std::vector<double> d(2 * m * m, 0.0);
    for (size_t i = 0; i < v.size(); ++i) d[2 * (i + 1)] = v[i]; // row 0, column i + 1
    return d;
}

std::vector<double> pathway_dipole_matrix(const config& cfg, size_t tensor, size_t spec, bool circular)
{
    const auto& comps = cfg.dipole_tensor_components();
    if (tensor >= comps.size() || spec >= comps[tensor].size())
        throw config_error("dipole.tensor_components has no entry for this pathway");
    const int64_t c = comps[tensor][spec];
    const auto& dirs = cfg.dipole_directions();
    const auto& ctrs = cfg.dipole_centers();
    const int sites = cfg.system().states;
    if ((int64_t)dirs.size() < sites) throw config_error("dipole.directions needs one direction per site");
    std::vector<double> v(sites);
    for (int i = 0; i < sites; ++i) {
        if (c < 0 || c >= (int64_t)dirs[i].size()) throw config_error("dipole.tensor_components out of range");
        double d = dirs[i][c];
        if (circular) { // (center x direction)[c], dipole_matrix.cpp:14-25
            if (dirs[i].size() != 3 || ctrs[i].size() != 3 || c > 2)
                throw config_error("circular dichroism needs 3-vectors in dipole.centers and dipole.directions");
            const std::vector<double>& a = ctrs[i];
            const std::vector<double>& b = dirs[i];
            const double cx[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
            d = cx[c];
        }
        v[i] = d * cfg.dipole_strengths()[i];
    }
    std::vector<double> d = dipole_matrix(v);
    if (spec == 1) { // the plus dipole of the pathway: the transpose
        const size_t m = v.size() + 1;
        std::vector<double> t(d.size());
        for (size_t i = 0; i < m; ++i)
            for (size_t j = 0; j < m; ++j) {
                t[2 * (j * m + i)] = d[2 * (i * m + j)];
                t[2 * (j * m + i) + 1] = d[2 * (i * m + j) + 1];
            }
        d.swap(t);
    }
    return d;
}

} // namespace heomhost
