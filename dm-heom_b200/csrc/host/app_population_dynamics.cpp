// app_population_dynamics.cpp -- population dynamics on one B200.
//
// Same command line and flow as dm-heom/src/app_population_dynamics.cpp:33-138:
//   heom_population_dynamics <runtime_config> <heom_config>
// parse -> hierarchy graph -> instance -> solver -> mask -> observers ->
// propagate with an observation every program.observe_steps steps.
//
// The runtime config replaces the reference's OpenCL config: a [cuda] section
// with device_index, rk4_scheme (product | horner | reference), ado_order
// (lex | reference) and use_graphs; an [opencl] section of a reference
// runtime config is accepted and ignored.
//
// Observers write the files named in program.observations with the headers of
// matrix_diagonal_observer.hpp:51-61, matrix_complete_observer.hpp,
// matrix_trace_observer.hpp:111-116, hierarchy_norm_observer.hpp:61-68 and
// hierarchy_complete_observer.hpp:58-70 (one line per observation: time, then the
// values), tab separated, numbers with 17 significant digits.
#include <chrono>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <sstream>

#include "heom_host.hpp"

using namespace heomhost;

namespace {

struct runtime_config {
    heom_options opt{};
};

runtime_config read_runtime_config(const std::string& path)
{
    runtime_config rc;
    heom_default_options(&rc.opt);
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
        if (eq == std::string::npos) continue;
        const std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
        if (section != "cuda") continue; // [opencl] and others: accepted, not used
        if (key == "device_index") rc.opt.device = (int32_t)parse_int(val);
        else if (key == "rk4_scheme") {
            if (val == "product") rc.opt.rk4_scheme = HEOM_RK4_PRODUCT;
            else if (val == "horner") rc.opt.rk4_scheme = HEOM_RK4_HORNER;
            else if (val == "reference") rc.opt.rk4_scheme = HEOM_RK4_REFERENCE;
            else throw config_error("cuda.rk4_scheme must be product, horner or reference");
        } else if (key == "ado_order") {
            if (val == "lex") rc.opt.ado_order = HEOM_ORDER_LEX;
            else if (val == "reference") rc.opt.ado_order = HEOM_ORDER_REFERENCE;
            else throw config_error("cuda.ado_order must be lex or reference");
        } else if (key == "use_graphs") rc.opt.use_graphs = parse_bool(val) ? 1 : 0;
        else throw config_error("unrecognised option 'cuda." + key + "'");
    }
    return rc;
}

std::string fmt(double v)
{
    char buf[40];
    std::snprintf(buf, sizeof buf, "%.17g", v);
    return buf;
}

const char kDelim = '\t';

bool whole_hierarchy(const std::string& type) { return type == "hierarchy_norm" || type == "hierarchy_complete"; }

void check(int rc)
{
    if (rc != 0) throw std::runtime_error(std::string("heom error: ") + heom_last_error());
}

struct file_observer {
    std::string type;
    std::ofstream out;
    int n;
    heom_handle* h;
    int64_t matrices;
    std::vector<double> buf;
    file_observer(const observation& o, int states, heom_handle* handle, const hierarchy_graph& g)
        : type(o.type), out(o.filename), n(states), h(handle), matrices(g.nodes())
    {
        if (!out.is_open()) throw std::runtime_error("file_observer_wrapper(): error: could not open output file: " + o.filename);
        out << "time";
        if (type == "hierarchy_norm") { // hierarchy_norm_observer.hpp:61-68: one column per ADO tuple
            const int64_t w = g.width();
            for (int64_t u = 0; u < matrices; ++u) {
                out << kDelim << '{';
                for (int64_t k = 0; k < w; ++k) out << (k ? ", " : "") << g.tuples()[u * w + k];
                out << '}';
            }
            buf.resize(matrices);
        } else if (type == "hierarchy_complete") { // hierarchy_complete_observer.hpp:58-70
            for (int64_t u = 0; u < matrices; ++u)
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < n; ++j)
                        for (int k = 0; k < 2; ++k)
                            out << kDelim << "mat_" << u << "_elem_" << i << "_" << j << (k == 0 ? "_real" : "_imag");
            buf.resize((size_t)matrices * n * n * 2);
        } else if (type == "matrix_diagonal") {
            for (int i = 0; i < n; ++i) out << kDelim << "site_" << i;
        } else if (type == "matrix_complete") {
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j)
                    for (int k = 0; k < 2; ++k) out << kDelim << "elem_" << i << "_" << j << (k == 0 ? "_real" : "_imag");
        } else if (type == "matrix_trace_id") {
            out << kDelim << "trace_real" << kDelim << "trace_imag";
        }
        out << '\n';
    }
    void observe(double time, const double* top)
    {
        out << fmt(time);
        if (type == "hierarchy_norm") {
            check(heom_hierarchy_norm(h, -1.0, buf.data()));
            for (double v : buf) out << kDelim << fmt(v);
        } else if (type == "hierarchy_complete") {
            check(heom_get_state(h, buf.data()));
            for (double v : buf) out << kDelim << fmt(v);
        } else if (type == "matrix_diagonal") {
            for (int i = 0; i < n; ++i) out << kDelim << fmt(top[(n + 1) * 2 * i]);
        } else if (type == "matrix_complete") {
            for (int q = 0; q < 2 * n * n; ++q) out << kDelim << fmt(top[q]);
        } else if (type == "matrix_trace_id") {
            double tr = 0.0, ti = 0.0;
            for (int i = 0; i < n; ++i) {
                tr += top[(n + 1) * 2 * i];
                ti += top[(n + 1) * 2 * i + 1];
            }
            out << kDelim << fmt(tr) << kDelim << fmt(ti);
        }
        out << '\n';
    }
};

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
        runtime_config rc = read_runtime_config(argv[1]);
        std::cout << "Parsing HEOM configuration from file: " << argv[2] << std::endl;
        heomhost::config cfg(argv[2]);
        bool per_observation = false; // observers that read the whole hierarchy
        for (const auto& o : cfg.observations()) {
            if (o.type != "matrix_diagonal" && o.type != "matrix_complete" && o.type != "matrix_trace_id" &&
                !whole_hierarchy(o.type))
                throw config_error("observation type " + o.type + " is not supported by this application");
            per_observation = per_observation || whole_hierarchy(o.type);
        }

        instance inst = make_instance(cfg.system());
        const int n = inst.sys.states;
        std::cout << "hierarchy: states " << n << ", width " << inst.width << ", depth " << inst.sys.depth
                  << ", matrices " << inst.matrices << std::endl;
        heom_instance_desc d = inst.desc();
        heom_handle* h = nullptr;
        check(heom_create(&d, &rc.opt, &h));
        std::unique_ptr<heom_handle, int (*)(heom_handle*)> guard(h, heom_destroy);

        hierarchy_graph g(inst.width, inst.sys.depth);
        std::vector<uint8_t> mask = make_mask(cfg.filtering_strategy(), g, inst.sys.matsubaras, cfg.filtering_first_layer());
        check(heom_set_mask(h, mask.data()));
        std::vector<double> top(2 * n * n);
        for (int q = 0; q < n * n; ++q) {
            top[2 * q] = cfg.rho_init()[q].real();
            top[2 * q + 1] = cfg.rho_init()[q].imag();
        }
        check(heom_set_top(h, top.data()));

        std::vector<std::unique_ptr<file_observer>> obs;
        for (const auto& o : cfg.observations()) obs.emplace_back(new file_observer(o, n, h, g));

        // flow tracking (population_dynamics_solver.hpp:141-150, 236-263): two
        // flow buffers handed to the derivative, zeroed at every step by the
        // stepping calls, their hierarchy norms taken after the step.  The
        // reference computes the norms but writes no file; with a
        // solver.flow_filename this application writes, at every observation,
        // the sum over ADOs of each buffer's norm for the last step.
        heom_buffer* flow_b[2] = {nullptr, nullptr};
        std::unique_ptr<heom_buffer, int (*)(heom_buffer*)> flow_a_guard(nullptr, heom_buffer_destroy);
        std::unique_ptr<heom_buffer, int (*)(heom_buffer*)> flow_b_guard(nullptr, heom_buffer_destroy);
        std::ofstream flow_out;
        std::vector<double> flow_norm(cfg.track_flows() ? inst.matrices : 0);
        if (cfg.track_flows()) {
            check(heom_buffer_create(h, &flow_b[0]));
            flow_a_guard.reset(flow_b[0]);
            check(heom_buffer_create(h, &flow_b[1]));
            flow_b_guard.reset(flow_b[1]);
            check(heom_set_flow_buffers(h, flow_b[0], flow_b[1]));
            if (!cfg.flow_filename().empty()) {
                flow_out.open(cfg.flow_filename());
                if (!flow_out.is_open()) throw std::runtime_error("could not open flow file: " + cfg.flow_filename());
                flow_out << "time" << kDelim << "flow_from_above_norm" << kDelim << "flow_from_below_norm" << '\n';
                per_observation = true; // the flows are read after every observation's steps
            }
        }
        auto observe_flows = [&](double time) {
            if (!flow_out.is_open()) return;
            flow_out << fmt(time);
            for (heom_buffer* b : flow_b) {
                check(heom_buffer_hierarchy_norm(h, b, flow_norm.data()));
                double sum = 0.0;
                for (double v : flow_norm) sum += v;
                flow_out << kDelim << fmt(sum);
            }
            flow_out << '\n';
        };

        const int64_t observe_steps = cfg.observe_steps();
        const int64_t iterations = cfg.steps() / observe_steps;
        const double dt = cfg.step_size();
        const int64_t chunk = std::max<int64_t>(1, std::min<int64_t>(iterations, 256));
        std::vector<double> tops((size_t)(chunk + 1) * 2 * n * n);
        for (auto& o : obs) o->observe(0.0, top.data()); // observer_list.observe(0.0)
        const auto ts = std::chrono::steady_clock::now();
        if (per_observation) {
            // every observation reads from the device: one stepping call per observation
            for (int64_t i = 1; i <= iterations; ++i) {
                check(heom_rk4_steps(h, dt, observe_steps));
                check(heom_get_top(h, top.data()));
                for (auto& o : obs) o->observe((double)(i * observe_steps) * dt, top.data());
                observe_flows((double)(i * observe_steps) * dt);
            }
        } else {
            for (int64_t i = 0; i < iterations; i += chunk) {
                const int64_t rows = std::min(chunk, iterations - i);
                check(heom_propagate(h, dt, rows * observe_steps, observe_steps, tops.data()));
                for (int64_t r = 1; r <= rows; ++r) {
                    const double time = (double)((i + r) * observe_steps) * dt;
                    for (auto& o : obs) o->observe(time, tops.data() + r * 2 * n * n);
                }
            }
        }
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - ts).count();
        const double updates = (double)inst.matrices * (double)(iterations * observe_steps);
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
