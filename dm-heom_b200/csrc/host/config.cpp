// config.cpp -- population_dynamics, linear_absorption and circular_dichroism
// configuration files.
//
// Reads the reference's INI files (dm-heom/src/heom/config.cpp:37-67,
// population_dynamics_config.cpp:24-26, linear_absorption_config.cpp:17-53,
// circular_dichroism_config.cpp:17-53,
// dipole_config_entries.cpp:19-41, config_base.cpp:32): "[section]"
// headers, "key=value" lines, '#' comments to the end of a line; values are
// noma/typa literals -- numbers, booleans, braced lists "{a, b}", braced
// matrices "{{a, b}, {c, d}}", complex numbers "(re, im)" or reals, and pair
// lists "{(type, file), ...}".  Validation follows config::check
// (config.cpp:73-175), population_dynamics_config::check (:32-41) and
// dipole_config_entries::check (:30-37); unit conversion follows
// config::post_process (config.cpp:182-191) (the dipole strengths stay in
// Debye: dipole_config_entries.cpp:39-41 leaves them unscaled).
#include <algorithm>
#include <cctype>
#include <cstdlib>
#include <fstream>
#include <set>
#include <sstream>

#include "heom_host.hpp"

namespace heomhost {

namespace {

std::string trim(const std::string& s)
{
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) ++a;
    while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
    return s.substr(a, b - a);
}

const std::set<std::string>& known_keys()
{
    static const std::set<std::string> k = {
        "program.task", "program.observations", "program.observe_steps",
        "filtering.strategy", "filtering.first_layer",
        "solver.stepper_type", "solver.step_size", "solver.steps", "solver.track_flows", "solver.flow_filename",
        "system.sites", "system.ado_depth", "system.hamiltonian",
        "baths.number", "baths.max_per_site", "baths.coupling", "baths.lambda", "baths.invnu", "baths.Omega",
        "baths.matsubaras", "baths.temperature"};
    return k;
}

// the keys each task adds (population_dynamics_config.cpp:24-26, dipole_config_entries.cpp:19-27)
const std::set<std::string>& task_keys(const std::string& task)
{
    static const std::set<std::string> pd = {"population_dynamics.rho_init"};
    static const std::set<std::string> la = {"dipole.directions", "dipole.strengths", "dipole.centers",
                                             "dipole.tensor_prefactors", "dipole.tensor_components"};
    static const std::set<std::string> none;
    return task == "population_dynamics" ? pd : (task == "linear_absorption" || task == "circular_dichroism") ? la : none;
}

bool any_task_key(const std::string& key)
{
    return task_keys("population_dynamics").count(key) || task_keys("linear_absorption").count(key);
}

const std::set<std::string>& observation_types()
{
    // observation_type.hpp:37-48
    static const std::set<std::string> k = {
        "matrix_diagonal", "matrix_complete", "matrix_complete_rate_kernel", "matrix_trace_id",
        "matrix_trace_linear_absorption", "matrix_trace_transient_absorption",
        "matrix_trace_static_fluorescence", "matrix_trace_two_dimensional_spectra",
        "hierarchy_norm", "hierarchy_complete"};
    return k;
}

std::vector<std::vector<std::string>> parse_matrix_items(const std::string& v)
{
    std::vector<std::vector<std::string>> rows;
    for (const std::string& r : split_braced(v)) rows.push_back(split_braced(r));
    return rows;
}

} // namespace

std::vector<std::string> split_braced(const std::string& s0)
{
    const std::string s = trim(s0);
    if (s.size() < 2 || s.front() != '{' || s.back() != '}')
        throw config_error("expected a braced list: " + s0);
    std::vector<std::string> items;
    const std::string body = s.substr(1, s.size() - 2);
    int depth = 0;
    std::string cur;
    for (char c : body) {
        if (c == '{' || c == '(') depth++;
        if (c == '}' || c == ')') depth--;
        if (depth < 0) throw config_error("unbalanced brackets in: " + s0);
        if (c == ',' && depth == 0) {
            items.push_back(trim(cur));
            cur.clear();
        } else {
            cur.push_back(c);
        }
    }
    if (depth != 0) throw config_error("unbalanced brackets in: " + s0);
    if (!trim(cur).empty() || !items.empty()) items.push_back(trim(cur));
    for (const std::string& it : items)
        if (it.empty()) throw config_error("empty list element in: " + s0);
    return items;
}

double parse_real(const std::string& s0)
{
    const std::string s = trim(s0);
    char* end = nullptr;
    const double v = std::strtod(s.c_str(), &end);
    if (s.empty() || *end != '\0') throw config_error("faulty value: not a real number: '" + s0 + "'");
    return v;
}

int64_t parse_int(const std::string& s0)
{
    const std::string s = trim(s0);
    char* end = nullptr;
    const long long v = std::strtoll(s.c_str(), &end, 10);
    if (s.empty() || *end != '\0') throw config_error("faulty value: not an integer: '" + s0 + "'");
    return v;
}

bool parse_bool(const std::string& s0)
{
    const std::string s = trim(s0);
    if (s == "true" || s == "1" || s == "yes" || s == "on") return true;
    if (s == "false" || s == "0" || s == "no" || s == "off") return false;
    throw config_error("faulty value: not a boolean: '" + s0 + "'");
}

complex_t parse_complex(const std::string& s0)
{
    const std::string s = trim(s0);
    if (!s.empty() && s.front() == '(') {
        if (s.back() != ')') throw config_error("faulty value: bad complex literal '" + s0 + "'");
        const std::string body = s.substr(1, s.size() - 2);
        const size_t c = body.find(',');
        if (c == std::string::npos) throw config_error("faulty value: bad complex literal '" + s0 + "'");
        return complex_t(parse_real(body.substr(0, c)), parse_real(body.substr(c + 1)));
    }
    return complex_t(parse_real(s), 0.0);
}

const std::string& config::raw(const std::string& key) const
{
    auto it = values_.find(key);
    if (it == values_.end()) throw config_error("the option '" + key + "' is required but missing");
    return it->second;
}

config::config(const std::string& path)
{
    std::ifstream f(path);
    if (f.fail()) throw config_error("could not open config file: " + path);
    std::string line, section;
    int lineno = 0;
    while (std::getline(f, line)) {
        ++lineno;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        line = trim(line);
        if (line.empty()) continue;
        if (line.front() == '[') {
            if (line.back() != ']') throw config_error("bad section header at line " + std::to_string(lineno));
            section = trim(line.substr(1, line.size() - 2));
            continue;
        }
        const size_t eq = line.find('=');
        if (eq == std::string::npos) throw config_error("expected key=value at line " + std::to_string(lineno));
        const std::string key = (section.empty() ? "" : section + ".") + trim(line.substr(0, eq));
        if (!known_keys().count(key) && !any_task_key(key)) throw config_error("unrecognised option '" + key + "'");
        if (values_.count(key)) throw config_error("option '" + key + "' cannot be specified more than once");
        values_[key] = trim(line.substr(eq + 1));
    }

    // program (config_base.cpp:32, config.cpp:39-40)
    task_ = raw("program.task");
    if (task_ != "population_dynamics" && task_ != "linear_absorption" && task_ != "circular_dichroism")
        throw config_error("program.task '" + task_ +
                           "' is not supported (population_dynamics, linear_absorption, circular_dichroism)");
    for (const auto& kv : values_)
        if (!known_keys().count(kv.first) && !task_keys(task_).count(kv.first))
            throw config_error("unrecognised option '" + kv.first + "'");
    for (const std::string& it : split_braced(raw("program.observations"))) {
        const std::string s = trim(it);
        if (s.size() < 2 || s.front() != '(' || s.back() != ')') throw config_error("bad observation entry: " + it);
        const std::string body = s.substr(1, s.size() - 2);
        const size_t c = body.find(',');
        if (c == std::string::npos) throw config_error("bad observation entry: " + it);
        observation o{trim(body.substr(0, c)), trim(body.substr(c + 1))};
        if (!observation_types().count(o.type)) throw config_error("unknown observation type: " + o.type);
        observations_.push_back(o);
    }
    observe_steps_ = parse_int(raw("program.observe_steps"));
    filtering_strategy_ = raw("filtering.strategy");
    if (filtering_strategy_ != "none" && filtering_strategy_ != "single_excitation")
        throw config_error("unknown filtering strategy: " + filtering_strategy_);
    filtering_first_layer_ = parse_int(raw("filtering.first_layer"));
    stepper_type_ = raw("solver.stepper_type");
    step_size_ = parse_real(raw("solver.step_size"));
    steps_ = parse_int(raw("solver.steps"));
    track_flows_ = parse_bool(raw("solver.track_flows"));
    flow_filename_ = raw("solver.flow_filename");

    // system / baths, config units
    const int64_t sites = parse_int(raw("system.sites"));
    const int64_t depth = parse_int(raw("system.ado_depth"));
    const auto hrows = parse_matrix_items(raw("system.hamiltonian"));
    for (const auto& r : hrows)
        for (const auto& v : r) {
            const complex_t z = parse_complex(v);
            h_flat_.push_back(z.real());
            h_flat_.push_back(z.imag());
        }
    const int64_t baths = parse_int(raw("baths.number"));
    const int64_t max_per_site = parse_int(raw("baths.max_per_site"));
    const auto crows = parse_matrix_items(raw("baths.coupling"));
    for (const auto& it : split_braced(raw("baths.lambda"))) lambda_.push_back(parse_real(it));
    for (const auto& it : split_braced(raw("baths.invnu"))) invnu_.push_back(parse_real(it));
    for (const auto& it : split_braced(raw("baths.Omega"))) omega_.push_back(parse_real(it));
    const int64_t matsubaras = parse_int(raw("baths.matsubaras"));
    const double temperature = parse_real(raw("baths.temperature"));

    // config::check (config.cpp:73-175)
    if (!(observe_steps_ > 0)) throw config_error("program.observe_steps must be > 0");
    if (filtering_strategy_ == "none" && filtering_first_layer_ != -1)
        throw config_error("filtering.first_layer must be -1, because it has no effect for filtering_strategy = none");
    if (filtering_strategy_ == "single_excitation" && !(filtering_first_layer_ >= 0))
        throw config_error("filtering.first_layer must be greater or equal to zero for filtering.strategy = single excitation filter");
    if (depth < filtering_first_layer_) throw config_error("filtering.first_layer cannot be larger than system_ado_depth");
    if (!(step_size_ > 0.0)) throw config_error("solver.step_size must be > 0");
    if (!(steps_ > 0)) throw config_error("solver.steps must be > 0");
    if (steps_ % observe_steps_ != 0)
        throw config_error("there's a remainder when dividing solver.steps by program.observe_steps");
    if (!(sites > 0)) throw config_error("system.sites must be > 0");
    if (!(depth > 0)) throw config_error("system.ado_depth must be > 0");
    if ((int64_t)hrows.size() != sites)
        throw config_error("system.hamiltonien must be a system.sites by system.sites matrix");
    for (const auto& r : hrows)
        if ((int64_t)r.size() != sites) throw config_error("system.hamiltonien must be a system.sites by system.sites matrix");
    if ((int64_t)crows.size() != sites) throw config_error("baths.coupling must be a system.sites by baths_max_per_site_ matrix");
    for (const auto& r : crows) {
        if ((int64_t)r.size() != max_per_site)
            throw config_error("baths.coupling must be a system.sites by baths_max_per_site_ matrix");
        for (const auto& v : r) coupling_.push_back((int32_t)parse_int(v));
    }
    if (stepper_type_ != "rk_rk4")
        throw config_error("solver.stepper_type '" + stepper_type_ + "' is not supported (rk_rk4 only)");

    desc_.sites = (int32_t)sites;
    desc_.ado_depth = (int32_t)depth;
    desc_.hamiltonian = h_flat_.data();
    desc_.baths = (int32_t)baths;
    desc_.baths_max_per_site = (int32_t)max_per_site;
    desc_.baths_coupling = coupling_.data();
    desc_.lambda = lambda_.data();
    desc_.invnu = invnu_.data();
    desc_.omega = omega_.data();
    desc_.matsubaras = (int32_t)matsubaras;
    desc_.temperature = temperature;
    if ((int64_t)lambda_.size() != baths) throw config_error("baths.lambda must have a length of baths.number");
    if ((int64_t)invnu_.size() != baths) throw config_error("baths.invnu must have a length of baths.number");
    if ((int64_t)omega_.size() != baths) throw config_error("baths.Omega must have a length of baths.number");
    sys_ = system_from_desc(desc_);
    sys_.depth = (int32_t)depth;
    validate_system(sys_);

    if (task_ == "population_dynamics") {
        // population_dynamics.rho_init (population_dynamics_config.cpp:32-41)
        const auto rrows = parse_matrix_items(raw("population_dynamics.rho_init"));
        if ((int64_t)rrows.size() != sites)
            throw config_error("population_dynamics.rho_init must be a system.sites by system.sites matrix");
        for (const auto& r : rrows) {
            if ((int64_t)r.size() != sites)
                throw config_error("population_dynamics.rho_init must be a system.sites by system.sites matrix");
            for (const auto& v : r) rho_init_.push_back(parse_complex(v));
        }
    } else {
        // dipole entries (dipole_config_entries.cpp:19-37)
        auto vectors = [&](const std::string& key) {
            std::vector<std::vector<double>> out;
            for (const auto& r : parse_matrix_items(raw(key))) {
                out.emplace_back();
                for (const auto& v : r) out.back().push_back(parse_real(v));
            }
            return out;
        };
        dipole_directions_ = vectors("dipole.directions");
        dipole_centers_ = vectors("dipole.centers");
        for (const auto& v : split_braced(raw("dipole.strengths"))) dipole_strengths_.push_back(parse_real(v));
        for (const auto& v : split_braced(raw("dipole.tensor_prefactors")))
            dipole_tensor_prefactors_.push_back(parse_real(v));
        for (const auto& r : parse_matrix_items(raw("dipole.tensor_components"))) {
            dipole_tensor_components_.emplace_back();
            for (const auto& v : r) dipole_tensor_components_.back().push_back(parse_int(v));
        }
        if (dipole_directions_.size() != dipole_strengths_.size() || dipole_directions_.size() != dipole_centers_.size())
            throw config_error("dipole.directions, dipole.strengths and dipole.centers must have the same size");
        if (dipole_tensor_prefactors_.size() != dipole_tensor_components_.size())
            throw config_error("dipole.tensor_prefactors and dipole.tensor_components must have the same size");
    }
}

} // namespace heomhost
