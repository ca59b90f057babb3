// app_linear_absorption.cpp -- linear absorption (and, built with
// HEOM_CIRCULAR_DICHROISM, circular dichroism) on one B200.
//
// Same command line and flow as dm-heom/src/app_linear_absorption.cpp:39-183:
//   heom_linear_absorption <runtime_config> <heom_config>
// and dm-heom/src/app_circular_dichroism.cpp:36-174:
//   heom_circular_dichroism <runtime_config> <heom_config>
// which differs in D-: the magnetic dipole (center x direction,
// dipole_matrix.hpp:43-48, 60-64), and applies no filtering mask.
// For every dipole tensor component t (dipole.tensor_prefactors /
// dipole.tensor_components): the state system with a ground state
// (sites_to_states with_ground_state), the top |g><g| with every other ADO
// zero, D+_t applied from the left to the hierarchy (hierarchy_mmult_left),
// then RK4 propagation with the trace tr(D-_t rho_top) observed every
// program.observe_steps steps (matrix_trace_observer.hpp:127-160; D-_t
// scaled by the tensor prefactor, dipole_matrix.hpp:67-72).  The traces,
// summed over the components in their order and divided by their count
// (matrix_trace_observer.hpp:45-63), go to the file of the first
// program.observations entry: "time trace_real trace_imag", tab separated,
// 17 significant digits.
//
// The components are independent propagations of the same hierarchy and run
// as the instances of one batch handle (one stage launch per RK4 stage for
// all of them).  At t = 0 only the top is non-zero, so D+ applied to the
// hierarchy is D+ applied to the top, done on the host.  The runtime config
// is that of heom_population_dynamics ([cuda] device_index, rk4_scheme,
// ado_order, use_graphs; [opencl] accepted and ignored).
#include <chrono>
#include <complex>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <memory>

#include "heom_host.hpp"

using namespace heomhost;

namespace {

#ifdef HEOM_CIRCULAR_DICHROISM
constexpr bool kCircular = true;
const char* const kTask = "circular_dichroism";
#else
constexpr bool kCircular = false;
const char* const kTask = "linear_absorption";
#endif

void check(int rc)
{
    if (rc != 0) throw std::runtime_error(std::string("heom error: ") + heom_last_error());
}

std::string fmt(double v)
{
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    return buf;
}

heom_options read_runtime_options(const std::string& path)
{
    heom_options o;
    heom_default_options(&o);
    std::ifstream f(path);
    if (f.fail()) throw config_error("could not open runtime config file: " + path);
    std::string line, section;
    auto trim = [](std::string s) {
        while (!s.empty() && isspace((unsigned char)s.back())) s.pop_back();
        size_t a = 0;
        while (a < s.size() && isspace((unsigned char)s[a])) ++a;
        return s.substr(a);
    };
    while (std::getline(f, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        line = trim(line);
        if (line.empty()) continue;
        if (line.front() == '[') {
            section = trim(line.substr(1, line.size() - 2));
            continue;
        }
        const size_t eq = line.find('=');
        if (eq == std::string::npos || section != "cuda") continue;
        const std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
        if (key == "device_index") o.device = (int32_t)parse_int(val);
        else if (key == "rk4_scheme") {
            if (val == "product") o.rk4_scheme = HEOM_RK4_PRODUCT;
            else if (val == "horner") o.rk4_scheme = HEOM_RK4_HORNER;
            else if (val == "reference") o.rk4_scheme = HEOM_RK4_REFERENCE;
            else throw config_error("cuda.rk4_scheme must be product, horner or reference");
        } else if (key == "ado_order") {
            if (val == "lex") o.ado_order = HEOM_ORDER_LEX;
            else if (val == "reference") o.ado_order = HEOM_ORDER_REFERENCE;
            else throw config_error("cuda.ado_order must be lex or reference");
        } else if (key == "use_graphs") o.use_graphs = parse_bool(val) ? 1 : 0;
        else throw config_error("unrecognised option 'cuda." + key + "'");
    }
    return o;
}

using cplx = std::complex<double>;

// tr(D rho) of two states x states matrices (interleaved), as ublas::prod then the diagonal sum
cplx trace_of_product(const std::vector<double>& d, const double* rho, int m)
{
    cplx tr(0.0, 0.0);
    for (int i = 0; i < m; ++i) {
        cplx e(0.0, 0.0);
        for (int k = 0; k < m; ++k)
            e += cplx(d[2 * (i * m + k)], d[2 * (i * m + k) + 1]) * cplx(rho[2 * (k * m + i)], rho[2 * (k * m + i) + 1]);
        tr += e;
    }
    return tr;
}

} // namespace

int main(int argc, char* argv[])
{
    const auto t0 = std::chrono::steady_clock::now();
    try {
        if (argc != 3) {
            std::cerr << "usage: " << argv[0] << " <runtime_config> <heom_config>" << std::endl;
            return -1;
        }
        std::cout << "Parsing runtime configuration from file: " << argv[1] << std::endl;
        heom_options opt = read_runtime_options(argv[1]);
        std::cout << "Parsing HEOM configuration from file: " << argv[2] << std::endl;
        heomhost::config cfg(argv[2]);
        if (cfg.task() != kTask) throw config_error("wrong program_task for this application");
        const std::string& out_name = cfg.observations().front().filename;
        std::ofstream out(out_name);
        if (out.fail()) throw std::runtime_error("Error: could not open output file: " + out_name);

        const system_params sys = state_system(cfg.system(), sites_to_states_mode::with_ground_state);
        instance inst = make_instance(sys);
        const int m = sys.states;
        const size_t K = cfg.dipole_tensor_prefactors().size();
        if (K == 0) throw config_error("dipole.tensor_prefactors is empty");
        std::cout << "hierarchy: states " << m << " (ground state + " << m - 1 << " sites), width " << inst.width
                  << ", depth " << sys.depth << ", matrices " << inst.matrices << ", tensor components " << K
                  << std::endl;

        // per component: top = D+ |g><g| (column 0 of D+ in column 0), D- scaled by the prefactor
        std::vector<std::vector<double>> tops0(K), dminus(K);
        for (size_t k = 0; k < K; ++k) {
            const std::vector<double> dplus = pathway_dipole_matrix(cfg, k, 1);
            tops0[k].assign(2 * m * m, 0.0);
            for (int i = 0; i < m; ++i) {
                tops0[k][2 * (i * m)] = dplus[2 * (i * m)];
                tops0[k][2 * (i * m) + 1] = dplus[2 * (i * m) + 1];
            }
            dminus[k] = pathway_dipole_matrix(cfg, k, 0, kCircular);
            const double pf = cfg.dipole_tensor_prefactors()[k]; // pathway sign plus
            for (double& v : dminus[k]) v *= pf;
        }

        std::vector<heom_instance_desc> descs(K, inst.desc());
        heom_handle* h = nullptr;
        check(heom_create_batch(descs.data(), (int32_t)K, &opt, &h));
        std::unique_ptr<heom_handle, int (*)(heom_handle*)> guard(h, heom_destroy);

        if (!kCircular) { // the circular-dichroism application sets no mask
            hierarchy_graph g(inst.width, sys.depth);
            const std::vector<uint8_t> mask1 =
                make_mask(cfg.filtering_strategy(), g, sys.matsubaras, cfg.filtering_first_layer());
            std::vector<uint8_t> mask;
            for (size_t k = 0; k < K; ++k) mask.insert(mask.end(), mask1.begin(), mask1.end());
            check(heom_set_mask(h, mask.data()));
        }

        for (size_t k = 0; k < K; ++k) check(heom_set_instance_top(h, (int32_t)k, tops0[k].data()));

        const int64_t observe_steps = cfg.observe_steps();
        const int64_t iterations = cfg.steps() / observe_steps;
        const double dt = cfg.step_size();
        const size_t row = (size_t)K * 2 * m * m;
        out << "time\ttrace_real\ttrace_imag\n";
        auto write_row = [&](double time, const double* tops) {
            cplx sum(0.0, 0.0);
            for (size_t k = 0; k < K; ++k) sum += trace_of_product(dminus[k], tops + k * 2 * m * m, m);
            out << fmt(time) << '\t' << fmt(sum.real() / (double)K) << '\t' << fmt(sum.imag() / (double)K) << '\n';
        };
        const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(iterations, 256));
        std::vector<double> tops((size_t)(chunk + 1) * row);
        const auto ts = std::chrono::steady_clock::now();
        for (int64_t i = 0; i < iterations; i += chunk) {
            const int64_t rows = std::min(chunk, iterations - i);
            check(heom_propagate(h, dt, rows * observe_steps, observe_steps, tops.data()));
            if (i == 0) write_row(0.0, tops.data());
            for (int64_t r = 1; r <= rows; ++r) write_row((double)((i + r) * observe_steps) * dt, tops.data() + r * row);
        }
        out << std::flush;
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
        const double updates = (double)inst.matrices * K * (double)(iterations * observe_steps);
        std::cout << "-------------------- Solver Runtime Summary ----------------\n"
                  << "steps: " << iterations * observe_steps << ", propagation time: " << secs << " s, "
                  << "ADO-updates/s: " << updates / secs << "\n"
                  << "kernel launches: " << heom_kernel_launches(h) << std::endl;
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << std::endl;
        return -1;
    }
    std::cout << "main(): application runtime: "
              << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() << " s" << std::endl;
    return 0;
}
