// host_capi.cpp -- C ABI of the host set-up (graph, tables, config, masks).
#include <cstring>
#include <memory>

#include "heom_host.hpp"

using namespace heomhost;

struct heom_tables {
    instance inst;
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
