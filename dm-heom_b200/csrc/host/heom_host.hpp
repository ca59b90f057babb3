// heom_host.hpp -- host side of the B200 HEOM propagator (C++17, no Boost).
//
// Mirrors the reference classes that feed the heom_ode path:
//   hierarchy_graph   dm-heom/include/heom/hierarchy_graph.hpp:29-95
//   instance          dm-heom/include/heom/instance.hpp:27-215
//   config            dm-heom/include/heom/config.hpp:30-152 and
//                     population_dynamics_config (population_dynamics_config.cpp:17-53)
#pragma once

#include <complex>
#include <cstdint>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "heom_b200.h"

namespace heomhost {

using complex_t = std::complex<double>;

constexpr double h_bar = 1.05457148e-34;                                       // constants.hpp:22
constexpr double k_b = 1.380650239684840458953781387048428305608616777679979316e-23; // :23
constexpr double invcm_to_joule = 1.986456217327470903861498336971100097137908380913187891e-23; // :24
constexpr int max_pade = 10;                                                    // :31
extern const long double heom_eta_pade[100];
extern const long double heom_xi_pade[100];
constexpr int32_t invalid_uid = -2;                                             // hierarchy_graph.cpp:24

struct config_error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// ---------------------------------------------------------------- graph --
// Nodes are the tuples n in N^width with |n| <= depth, numbered layer by
// layer as the reference does (hierarchy_graph.cpp:57-117).
class hierarchy_graph {
public:
    hierarchy_graph(int64_t width, int64_t depth);
    int64_t width() const { return width_; }
    int64_t depth() const { return depth_; }
    int64_t nodes() const { return nodes_; }
    int32_t first_non_plus_uid() const { return first_non_plus_; }
    const std::vector<int32_t>& tuples() const { return tuples_; } // [nodes][width]
    const std::vector<int32_t>& plus() const { return plus_; }
    const std::vector<int32_t>& minus() const { return minus_; }
    const std::vector<int64_t>& nodes_per_depth() const { return nodes_per_depth_; }
    // position of a tuple in ascending lexicographic order (a bijection onto 0..nodes-1)
    int64_t lex_rank(const int32_t* t) const;

private:
    int64_t width_, depth_, nodes_;
    int32_t first_non_plus_;
    std::vector<int32_t> tuples_, plus_, minus_;
    std::vector<int64_t> nodes_per_depth_;
    std::vector<std::vector<int64_t>> binom_;
};

int64_t binomial(int64_t n, int64_t k);
// partitions of n into at most s parts in the reference's order
// (integer_partition.cpp:41-106): ascending lexicographic order of the
// non-increasing part sequences; each row padded with zeros to s entries
std::vector<int32_t> integer_partitions(int32_t n, int32_t s);

// ------------------------------------------------------------- instance --
struct system_params {         // SI units, after config post_process
    int32_t states = 0;        // identity sites -> states
    int32_t depth = 0;
    std::vector<complex_t> hamiltonian; // [N*N] J
    int32_t baths = 0;
    int32_t baths_per_state = 0;
    std::vector<int32_t> coupling;      // [N * baths_per_state]
    std::vector<double> lambda;         // J
    std::vector<double> invnu;          // s
    std::vector<double> omega;          // rad/s
    int32_t matsubaras = 0;
    double temperature = 0.0;           // K
};

// host tables in the reference layouts (instance.hpp:202-214)
struct instance {
    system_params sys;
    int64_t matrices = 0;
    int32_t width = 0;
    int32_t first_non_plus = 0;
    std::vector<int32_t> tuples, plus, minus;
    std::vector<double> hamiltonian;   // [N*N*2]
    std::vector<double> pf_same_sum;   // [matrices*2]
    std::vector<double> pf_same, pf_circ, cbk, cbk_sqrt;

    heom_instance_desc desc() const;
};

// instance.cpp:25-71 + precompute_baths_input (:155-273)
instance make_instance(const system_params& sys);

// derivatives of the bath tables for the adjoint: index 0 = lambda of every
// bath together (per J), 1 = gamma = 1/invnu of every bath together (per 1/s)
struct bath_derivs {
    std::vector<double> pf_same[2], pf_circ[2], cbk[2]; // layouts of instance::pf_same, pf_circ, cbk
};
bath_derivs bath_derivatives(const system_params& sys);
system_params system_from_desc(const heom_system_desc& d); // config units -> SI (config.cpp:182-191)
void validate_system(const system_params& s);              // config.cpp:117-174 subset

// --------------------------------------------------------------- config --
struct observation {
    std::string type;
    std::string filename;
};

// An INI file with the reference's sections and literals
// ([program] [filtering] [solver] [system] [baths], then [population_dynamics]
// or [dipole] by program.task).
class config {
public:
    explicit config(const std::string& path);
    config(const config&) = delete; // system_desc() points into this object
    config& operator=(const config&) = delete;
    const std::string& task() const { return task_; }
    const std::vector<observation>& observations() const { return observations_; }
    int64_t observe_steps() const { return observe_steps_; }
    const std::string& filtering_strategy() const { return filtering_strategy_; }
    int64_t filtering_first_layer() const { return filtering_first_layer_; }
    const std::string& stepper_type() const { return stepper_type_; }
    double step_size() const { return step_size_; }
    int64_t steps() const { return steps_; }
    bool track_flows() const { return track_flows_; }
    const std::string& flow_filename() const { return flow_filename_; }
    // configuration values in config units (cm^-1, fs)
    const heom_system_desc& system_desc() const { return desc_; }
    const system_params& system() const { return sys_; }   // SI
    const std::vector<complex_t>& rho_init() const { return rho_init_; }
    // dipole entries (linear_absorption; dipole_config_entries.hpp:41-54)
    const std::vector<std::vector<double>>& dipole_directions() const { return dipole_directions_; }
    const std::vector<std::vector<double>>& dipole_centers() const { return dipole_centers_; }
    const std::vector<double>& dipole_strengths() const { return dipole_strengths_; }
    const std::vector<double>& dipole_tensor_prefactors() const { return dipole_tensor_prefactors_; }
    const std::vector<std::vector<int64_t>>& dipole_tensor_components() const { return dipole_tensor_components_; }
    // raw key lookup ("section.key")
    bool has(const std::string& key) const { return values_.count(key) != 0; }
    const std::string& raw(const std::string& key) const;

private:
    std::map<std::string, std::string> values_;
    std::string task_;
    std::vector<observation> observations_;
    int64_t observe_steps_ = 0;
    std::string filtering_strategy_;
    int64_t filtering_first_layer_ = -1;
    std::string stepper_type_;
    double step_size_ = 0.0;
    int64_t steps_ = 0;
    bool track_flows_ = false;
    std::string flow_filename_;
    heom_system_desc desc_{};
    std::vector<double> h_flat_, lambda_, invnu_, omega_;
    std::vector<int32_t> coupling_;
    system_params sys_;
    std::vector<complex_t> rho_init_;
    std::vector<std::vector<double>> dipole_directions_, dipole_centers_;
    std::vector<double> dipole_strengths_, dipole_tensor_prefactors_;
    std::vector<std::vector<int64_t>> dipole_tensor_components_;
};

// ------------------------------------------------------------- spectra --
enum class sites_to_states_mode { identity, with_ground_state };
// sites_to_states.cpp:16-28 (states), :44-55 (H: ground state row and column
// zero), :131-142 (coupling: the ground state couples to no bath)
system_params state_system(const system_params& sites, sites_to_states_mode mode);
// dipole_matrix.cpp:105-131 (with_ground_state): D(0, i+1) = v_i, every other
// entry zero; row-major states x states complex, interleaved
std::vector<double> dipole_matrix(const std::vector<double>& dipole_vector);
// dipole_matrix.hpp:30-58 for the pseudo pathway of linear absorption and
// circular dichroism (dipole_pseudo_pathway.hpp:22-27: {minus, left},
// {plus, left}): v_i = directions[i][component] * strengths[i] with component
// = tensor_components[tensor][spec], or for the magnetic dipole (circular)
// v_i = (centers[i] x directions[i])[component] * strengths[i]
// (dipole_matrix.hpp:43-48); spec 1 (plus) is the transpose
std::vector<double> pathway_dipole_matrix(const config& cfg, size_t tensor, size_t spec, bool circular = false);

// literal parsing (noma/typa-style values)
std::vector<std::string> split_braced(const std::string& s); // "{a, {b}, (c, d)}" -> items
double parse_real(const std::string& s);
int64_t parse_int(const std::string& s);
bool parse_bool(const std::string& s);
complex_t parse_complex(const std::string& s);

// hierarchy mask (dm-heom/src/heom/hierarchy_mask.cpp:20-110)
std::vector<uint8_t> make_mask(const std::string& strategy, const hierarchy_graph& g,
                               int32_t matsubaras, int64_t first_layer);

// records the calling thread's last error for heom_last_error()
int set_error(int code, const std::string& msg);

} // namespace heomhost
