// shock_params_from_ini: the config.ini keys of SHOCK's hot path.
//
// SHOCK reads its configuration with the iniparser it ships
// (src/iniparser.c:555-720, called from src/Import.c:17-275), and this reader
// follows the same rules for the keys the path consumes:
//   - a physical line loses its trailing white space; one that then ends in
//     a backslash continues on the next line (the backslash dropped);
//   - a line of more than 1022 characters (a continued line counted from
//     its start), or a last line without a newline, makes iniparser reject
//     the whole file (SHOCK then stops), and this reader too;
//   - after stripping: empty lines and lines starting with ';' or '#' are
//     skipped; "[name]" (first '[' and last ']') opens section name (up to
//     the first ']', stripped, lower case);
//   - "key = value": the key is everything before the first '=', stripped
//     and lower case; a value starting with '"' or '\'' runs to the next
//     such quote, any other value to the first ';' or '#', stripped; an
//     empty or missing value is the empty string; a later line with the
//     same key replaces the earlier one; other lines are ignored;
//   - numbers are read as iniparser's getters read them: doubles with
//     atof (an empty value is 0), integers with strtol in base 0
//     (TimeOrder), booleans true when the value starts with y/Y/t/T/1 and
//     false with n/N/f/F/0 (otherwise the field keeps its value).
// Keys missing from the file leave their fields unchanged, as do all other
// fields of *p (grid sizes, dimension and order come from the mesh and the
// build in SHOCK, so the caller sets them).
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

// iniparser's value of one "key = value" line (the part after the first
// '='): quoted up to the next quote of the same kind, else up to the first
// comment character, stripped
std::string ini_value(const std::string &rest)
{
    std::string v = trim(rest);
    if (!v.empty() && (v[0] == '"' || v[0] == '\'')) {
        const size_t e = v.find(v[0], 1);
        if (e == 1) return "";                                 // "" or ''
        if (e != std::string::npos || v.size() > 1) return trim(v.substr(1, e == std::string::npos ? e : e - 1));
    }
    const size_t c = v.find_first_of(";#");
    return trim(c == std::string::npos ? v : v.substr(0, c));
}

}  // namespace

extern "C" int shock_params_from_ini(const char *path, shock_params *p)
{
    if (!path || !p) return shock::report_error(SHOCK_EINVAL, "null argument");
    FILE *f = std::fopen(path, "r");
    if (!f) return shock::report_error(SHOCK_EINVAL, "cannot open %s", path);
    std::map<std::string, std::string> kv;   // "section:key" -> value
    std::string section, logical;
    char buf[1025];
    int lineno = 0;
    bool ok = true;
    while (std::fgets(buf, sizeof buf, f)) {
        lineno++;
        std::string raw(buf);
        if (raw.size() <= 1 && logical.empty()) continue;      // a bare newline
        // iniparser reads a line into 1023 characters after what the previous
        // lines of a continued line left, its newline included
        if (raw.back() != '\n' || raw.size() + logical.size() > 1023) {
            ok = false;                                        // too long, or no newline at the end
            break;
        }
        size_t end = raw.size();
        while (end > 0 && std::isspace((unsigned char)raw[end - 1])) end--;
        raw.resize(end);
        if (!raw.empty() && raw.back() == '\\') {              // continued on the next line
            raw.pop_back();
            logical += raw;
            continue;
        }
        std::string s = trim(logical + raw);
        logical.clear();
        if (s.empty() || s[0] == ';' || s[0] == '#') continue;
        if (s[0] == '[' && s.back() == ']') {
            const std::string name = s.substr(1, s.find(']') - 1);
            if (!name.empty()) section = lower(trim(name));    // "[]" leaves the section as it was
            continue;
        }
        const size_t eq = s.find('=');
        if (eq == std::string::npos || eq == 0) continue;      // iniparser: syntax error, line ignored
        kv[section + ":" + lower(trim(s.substr(0, eq)))] = ini_value(s.substr(eq + 1));
    }
    std::fclose(f);
    if (!ok)
        return shock::report_error(SHOCK_EINVAL,
                                   "%s line %d: longer than 1022 characters or without a newline at the end of the "
                                   "file; SHOCK's iniparser rejects the file",
                                   path, lineno);

    auto num = [&](const char *k, double &dst) {
        auto it = kv.find(k);
        if (it != kv.end()) dst = std::atof(it->second.c_str());
    };
    auto boolean = [&](const char *k, int &dst) {
        auto it = kv.find(k);
        if (it != kv.end()) dst = to_bool(it->second, dst);
    };
    auto it = kv.find("numerics:timeorder");
    if (it != kv.end()) p->time_order = (int)std::strtol(it->second.c_str(), nullptr, 0);
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
