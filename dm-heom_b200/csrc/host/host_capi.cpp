// host_capi.cpp -- C ABI of the host set-up (graph, tables, config, masks).
#include <cstring>
#include <fstream>
#include <memory>

#include "heom_host.hpp"

using namespace heomhost;

struct heom_tables {
    instance inst;
    std::vector<double> state; // hierarchy read from an instance file (empty: none)
    double time = 0.0;
};

struct heom_config {
    std::unique_ptr<heomhost::config> cfg;
};

namespace {
template <typename F>
int guarded(F&& f)
{
    try {
        return f();
    } catch (const config_error& e) {
        return set_error(HEOM_E_CONFIG, e.what());
    } catch (const std::bad_alloc&) {
        return set_error(HEOM_E_NOMEM, "host allocation failed");
    } catch (const std::exception& e) {
        return set_error(HEOM_E_ARG, e.what());
    }
}
} // namespace

extern "C" {

int heom_tables_build(const heom_system_desc* sys, heom_tables** out)
{
    if (!sys || !out) return set_error(HEOM_E_ARG, "NULL argument");
    *out = nullptr;
    return guarded([&] {
        std::unique_ptr<heom_tables> t(new heom_tables());
        t->inst = make_instance(system_from_desc(*sys));
        *out = t.release();
        return 0;
    });
}

int heom_tables_view(const heom_tables* t, heom_instance_desc* view)
{
    if (!t || !view) return set_error(HEOM_E_ARG, "NULL argument");
    *view = t->inst.desc();
    return 0;
}

void heom_tables_free(heom_tables* t) { delete t; }

int heom_create_from_system(const heom_system_desc* sys, const heom_options* opt, heom_handle** out)
{
    heom_tables* t = nullptr;
    if (int rc = heom_tables_build(sys, &t)) return rc;
    heom_instance_desc d;
    heom_tables_view(t, &d);
    const int rc = heom_create(&d, opt, out);
    heom_tables_free(t);
    return rc;
}

int heom_bath_derivatives(const heom_system_desc* sys, int32_t theta, double* d_pf_same, double* d_pf_circ,
                          double* d_cbk)
{
    if (!sys || theta < 0 || theta > 1) return set_error(HEOM_E_ARG, "bad argument");
    return guarded([&] {
        const system_params sp = system_from_desc(*sys);
        validate_system(sp);
        const bath_derivs d = bath_derivatives(sp);
        if (d_pf_same) std::memcpy(d_pf_same, d.pf_same[theta].data(), d.pf_same[theta].size() * 8);
        if (d_pf_circ) std::memcpy(d_pf_circ, d.pf_circ[theta].data(), d.pf_circ[theta].size() * 8);
        if (d_cbk) std::memcpy(d_cbk, d.cbk[theta].data(), d.cbk[theta].size() * 8);
        return 0;
    });
}

// The reference's binary instance file (instance::write_file / read_file,
// instance.cpp:281-377, format version 1): the fields one after another in
// native layout, no padding -- int32 version, bool hierarchy_top_only, int32
// hierarchy and hamiltonian layouts, the sites_to_states mode (an int), double
// time, int32 first_non_plus_id, int64 states, matrices, matsubaras,
// baths_per_state, baths, ado_width, ado_depth, then the hierarchy (all ADOs,
// or the top only), H, tuples, plus, minus, pf_same_sum, pf_same, pf_circ,
// cbk, cbk_sqrt.  The bath coupling is not in the file.
} // extern "C"

namespace {
template <typename T>
void put(std::ofstream& f, const T& v)
{
    f.write(reinterpret_cast<const char*>(&v), sizeof v);
}
template <typename T>
void put_n(std::ofstream& f, const T* p, size_t n)
{
    f.write(reinterpret_cast<const char*>(p), n * sizeof(T));
}
template <typename T>
void get(std::ifstream& f, T& v)
{
    f.read(reinterpret_cast<char*>(&v), sizeof v);
}
template <typename T>
void get_n(std::ifstream& f, T* p, size_t n)
{
    f.read(reinterpret_cast<char*>(p), n * sizeof(T));
}
} // namespace

extern "C" {

int heom_instance_write(const heom_tables* t, const double* state, int32_t top_only, double time, const char* path)
{
    if (!t || !path) return set_error(HEOM_E_ARG, "NULL argument");
    return guarded([&] {
        const instance& in = t->inst;
        std::ofstream f(path, std::ios::out | std::ios::binary | std::ios::trunc);
        if (!f) throw config_error(std::string("could not open instance file for writing: ") + path);
        const int64_t N = in.sys.states, nodes = in.matrices, W = in.width, B = in.sys.baths, M = in.sys.matsubaras;
        put(f, int32_t(0));           // version V_1
        put(f, bool(top_only != 0));  // hierarchy_top_only
        put(f, int32_t(0));           // hierarchy layout VANILLA
        put(f, int32_t(0));           // hamiltonian layout VANILLA
        put(f, int(0));               // sites_to_states identity
        put(f, time);
        put(f, int32_t(in.first_non_plus));
        for (int64_t v : {N, nodes, M, (int64_t)in.sys.baths_per_state, B, W, (int64_t)in.sys.depth}) put(f, v);
        const size_t hsz = (size_t)(top_only ? 1 : nodes) * N * N * 2;
        std::vector<double> zero;
        if (!state) zero.assign(hsz, 0.0);
        put_n(f, state ? state : zero.data(), hsz);
        put_n(f, in.hamiltonian.data(), (size_t)N * N * 2);
        put_n(f, in.tuples.data(), (size_t)nodes * W);
        put_n(f, in.plus.data(), (size_t)nodes * W);
        put_n(f, in.minus.data(), (size_t)nodes * W);
        put_n(f, in.pf_same_sum.data(), (size_t)nodes * 2);
        put_n(f, in.pf_same.data(), (size_t)B * 2);
        put_n(f, in.pf_circ.data(), (size_t)B * 2);
        put_n(f, in.cbk.data(), (size_t)B * M * 2);
        put_n(f, in.cbk_sqrt.data(), (size_t)B * M);
        if (!f) throw config_error(std::string("writing the instance file failed: ") + path);
        return 0;
    });
}

int heom_instance_read(const char* path, const int32_t* coupling, heom_tables** out)
{
    if (!path || !out) return set_error(HEOM_E_ARG, "NULL argument");
    *out = nullptr;
    return guarded([&] {
        std::ifstream f(path, std::ios::in | std::ios::binary);
        if (!f) throw config_error(std::string("could not open instance file: ") + path);
        int32_t version = -1, hl = 0, ml = 0, fnp = 0;
        bool top_only = false;
        int sts = 0;
        double time = 0.0;
        int64_t N = 0, nodes = 0, M = 0, bps = 0, B = 0, W = 0, D = 0;
        get(f, version);
        get(f, top_only);
        get(f, hl);
        get(f, ml);
        get(f, sts);
        get(f, time);
        get(f, fnp);
        for (int64_t* v : {&N, &nodes, &M, &bps, &B, &W, &D}) get(f, *v);
        if (!f || version != 0) throw config_error("not an instance file of format version 1");
        if (hl != 0 || ml != 0 || sts != 0) throw config_error("instance file: unsupported layout or sites_to_states mode");
        if (N < 1 || N > 64 || nodes < 1 || nodes > INT32_MAX || M < 1 || B < 1 || bps < 1 || W != B * M || D < 1)
            throw config_error("instance file: inconsistent sizes");
        std::unique_ptr<heom_tables> t(new heom_tables());
        instance& in = t->inst;
        in.sys.states = (int32_t)N;
        in.sys.depth = (int32_t)D;
        in.sys.baths = (int32_t)B;
        in.sys.baths_per_state = (int32_t)bps;
        in.sys.matsubaras = (int32_t)M;
        in.matrices = nodes;
        in.width = (int32_t)W;
        in.first_non_plus = fnp;
        in.sys.coupling.resize((size_t)N * bps);
        if (coupling) {
            std::copy(coupling, coupling + N * bps, in.sys.coupling.begin());
        } else {
            if (bps != 1 || B != N) throw config_error("instance file: give the bath coupling (it is not in the file)");
            for (int64_t i = 0; i < N; ++i) in.sys.coupling[i] = (int32_t)i;
        }
        const size_t hsz = (size_t)(top_only ? 1 : nodes) * N * N * 2;
        t->state.assign((size_t)nodes * N * N * 2, 0.0);
        get_n(f, t->state.data(), hsz);
        in.hamiltonian.resize((size_t)N * N * 2);
        get_n(f, in.hamiltonian.data(), in.hamiltonian.size());
        in.tuples.resize((size_t)nodes * W);
        in.plus.resize((size_t)nodes * W);
        in.minus.resize((size_t)nodes * W);
        get_n(f, in.tuples.data(), in.tuples.size());
        get_n(f, in.plus.data(), in.plus.size());
        get_n(f, in.minus.data(), in.minus.size());
        in.pf_same_sum.resize((size_t)nodes * 2);
        get_n(f, in.pf_same_sum.data(), in.pf_same_sum.size());
        in.pf_same.resize((size_t)B * 2);
        in.pf_circ.resize((size_t)B * 2);
        in.cbk.resize((size_t)B * M * 2);
        in.cbk_sqrt.resize((size_t)B * M);
        get_n(f, in.pf_same.data(), in.pf_same.size());
        get_n(f, in.pf_circ.data(), in.pf_circ.size());
        get_n(f, in.cbk.data(), in.cbk.size());
        get_n(f, in.cbk_sqrt.data(), in.cbk_sqrt.size());
        if (!f) throw config_error("instance file is truncated");
        t->time = time;
        *out = t.release();
        return 0;
    });
}

int heom_tables_state(const heom_tables* t, double* state, double* time)
{
    if (!t || !state) return set_error(HEOM_E_ARG, "NULL argument");
    if (t->state.empty()) return set_error(HEOM_E_ARG, "these tables were not read from an instance file");
    std::copy(t->state.begin(), t->state.end(), state);
    if (time) *time = t->time;
    return 0;
}

int heom_tables_mask(const heom_tables* t, const char* strategy, int64_t first_layer, uint8_t* mask)
{
    if (!t || !strategy || !mask) return set_error(HEOM_E_ARG, "NULL argument");
    return guarded([&] {
        hierarchy_graph g(t->inst.width, t->inst.sys.depth);
        std::vector<uint8_t> m = make_mask(strategy, g, t->inst.sys.matsubaras, first_layer);
        std::memcpy(mask, m.data(), m.size());
        return 0;
    });
}

int heom_config_load(const char* path, heom_config** out)
{
    if (!path || !out) return set_error(HEOM_E_ARG, "NULL argument");
    *out = nullptr;
    return guarded([&] {
        std::unique_ptr<heom_config> c(new heom_config());
        c->cfg.reset(new heomhost::config(path));
        *out = c.release();
        return 0;
    });
}

void heom_config_free(heom_config* c) { delete c; }

int heom_config_system(const heom_config* c, heom_system_desc* view)
{
    if (!c || !view) return set_error(HEOM_E_ARG, "NULL argument");
    *view = c->cfg->system_desc();
    return 0;
}

int heom_config_rho_init(const heom_config* c, double* out)
{
    if (!c || !out) return set_error(HEOM_E_ARG, "NULL argument");
    const auto& r = c->cfg->rho_init();
    if (r.empty()) return set_error(HEOM_E_ARG, "the configuration has no population_dynamics.rho_init");
    for (size_t q = 0; q < r.size(); ++q) {
        out[2 * q] = r[q].real();
        out[2 * q + 1] = r[q].imag();
    }
    return 0;
}

int heom_config_get(const heom_config* c, const char* key, char* buf, size_t len)
{
    if (!c || !key || !buf || len == 0) return set_error(HEOM_E_ARG, "NULL argument");
    if (!c->cfg->has(key)) return set_error(HEOM_E_CONFIG, std::string("no such option: ") + key);
    const std::string& v = c->cfg->raw(key);
    if (v.size() + 1 > len) return set_error(HEOM_E_ARG, "buffer too small");
    std::memcpy(buf, v.c_str(), v.size() + 1);
    return 0;
}

} // extern "C"
