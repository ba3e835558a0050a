// shock_params_from_ini: the config.ini keys of SHOCK's hot path.
//
// SHOCK reads its configuration with iniparser (src/Import.c:36-238):
// sections in brackets, "key = value" lines, ';' or '#' starting a comment,
// section and key names matched without regard to case, booleans true when
// the value starts with y/Y/t/T/1.  This reader follows the same rules for
// the keys the path consumes and leaves every other field of *p unchanged
// (grid sizes, dimension and order come from the mesh and the build in
// SHOCK, so the caller sets them).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>

#include "internal.h"

namespace {

std::string lower(std::string s)
{
    for (auto &ch : s) ch = (char)std::tolower((unsigned char)ch);
    return s;
}

std::string trim(const std::string &s)
{
    size_t a = 0, b = s.size();
    while (a < b && std::isspace((unsigned char)s[a])) a++;
    while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
    return s.substr(a, b - a);
}

// iniparser_getboolean: y/Y/t/T/1 true, n/N/f/F/0 false, else the default
int to_bool(const std::string &v, int def)
{
    if (v.empty()) return def;
    const char c = v[0];
    if (c == 'y' || c == 'Y' || c == 't' || c == 'T' || c == '1') return 1;
    if (c == 'n' || c == 'N' || c == 'f' || c == 'F' || c == '0') return 0;
    return def;
}

}  // namespace

extern "C" int shock_params_from_ini(const char *path, shock_params *p)
{
    if (!path || !p) return shock::report_error(SHOCK_EINVAL, "null argument");
    FILE *f = std::fopen(path, "r");
    if (!f) return shock::report_error(SHOCK_EINVAL, "cannot open %s", path);
    std::map<std::string, std::string> kv;   // "section:key" -> value
    std::string section;
    char line[4096];
    while (std::fgets(line, sizeof line, f)) {
        std::string s = trim(line);
        if (s.empty() || s[0] == ';' || s[0] == '#') continue;
        if (s[0] == '[') {
            size_t e = s.find(']');
            section = lower(trim(s.substr(1, e == std::string::npos ? std::string::npos : e - 1)));
            continue;
        }
        size_t eq = s.find('=');
        if (eq == std::string::npos) continue;
        std::string key = lower(trim(s.substr(0, eq)));
        std::string val = s.substr(eq + 1);
        size_t c = val.find_first_of(";#");
        if (c != std::string::npos) val = val.substr(0, c);
        kv[section + ":" + key] = trim(val);
    }
    std::fclose(f);

    auto num = [&](const char *k, double &dst) {
        auto it = kv.find(k);
        if (it != kv.end() && !it->second.empty()) dst = std::strtod(it->second.c_str(), nullptr);
    };
    auto boolean = [&](const char *k, int &dst) {
        auto it = kv.find(k);
        if (it != kv.end()) dst = to_bool(it->second, dst);
    };
    double t = p->time_order;
    num("numerics:timeorder", t);
    p->time_order = (int)t;
    num("numerics:tau", p->tau);
    num("fluidproperties:mach", p->mach);
    num("fluidproperties:reynolds", p->reynolds);
    num("fluidproperties:prandtl", p->prandtl);
    num("fluidproperties:gamma", p->gamma);
    num("fluidproperties:r", p->gas_r);
    num("fluidproperties:t", p->t0);
    num("fluidproperties:l", p->l0);
    num("boundaryconditions:t_wall", p->t_wall);
    num("boundaryconditions:rho_inflow", p->rho_inflow);
    num("boundaryconditions:p_inflow", p->p_inflow);
    num("boundaryconditions:p_outflow", p->p_outflow);
    // inflow velocity (src/Import.c:233-235): angle of attack in degrees and
    // [InitializeValues] u0, SHOCK's defaults 0 and 1 for a missing one
    if (kv.count("boundaryconditions:aoa") || kv.count("initializevalues:u0")) {
        double aoa = 0.0, u0 = 1.0;
        num("boundaryconditions:aoa", aoa);
        num("initializevalues:u0", u0);
        const double pi = 3.14159265358979323846;
        p->u_inflow[0] = std::cos(aoa / 360 * 2 * pi) * u0;
        p->u_inflow[1] = std::sin(aoa / 360 * 2 * pi) * u0;
        p->u_inflow[2] = 0.0;
    }
    boolean("options:inviscid", p->inviscid);
    boolean("options:manufacturedsolution", p->mms);
    return SHOCK_OK;
}
