// Input files of the reference, read by its own rules (host code only).
//
//  dft.in   src/module_input.f90: lines are read as 100-character records
//           (put_input_in_character_array, :654-732), left-adjusted, cut at the first '#',
//           left-adjusted again, blank lines dropped.  getinput%<kind>(tag) takes the
//           first line whose first len(tag) characters are the tag and whose next
//           character is a blank, and list-directed-reads the value from columns
//           len(tag)+4 .. len(tag)+50 (:73-79 and the other input_* functions): the value
//           is expected after "tag = ".  Logicals are decided by the first character of
//           the first item, T/t or F/f (:386-427).
//  solute.in  src/module_solute.f90:36-50: a comment line, the site count, a comment
//           line, then one line per site: index, q, sigma, epsilon, x, y, z, Z.
//  mv_solute_to_center  src/module_solute.f90:146-187.
#include "../../include/mdft_b200.h"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "common.cuh"

using namespace mdft;

struct mdft_input {
    std::vector<std::string> lines;  // 100-character records after the reference's clean-up
};

namespace {

constexpr size_t kRec = 100;  // character(len=100) records

std::string adjustl_trim(const std::string &s) {
    size_t a = 0;
    while (a < s.size() && s[a] == ' ') ++a;
    size_t b = s.size();
    while (b > a && s[b - 1] == ' ') --b;
    return s.substr(a, b - a);
}

// The value field of `tag` on line `l`: columns len(tag)+4 .. len(tag)+50 (1-based) of the
// blank-padded 100-character record; false when the line does not carry the tag.
bool value_field(const std::string &l, const char *tag, std::string *field) {
    const size_t j = std::strlen(tag);
    std::string rec = l;
    rec.resize(kRec, ' ');
    if (j == 0 || j >= kRec) return false;
    if (rec.compare(0, j, tag) != 0 || rec[j] != ' ') return false;
    const size_t a = j + 3, b = std::min(kRec, j + 50);
    *field = a < b ? rec.substr(a, b - a) : std::string();
    return true;
}

const std::string *find_tag(const mdft_input *in, const char *tag, std::string *field) {
    for (const auto &l : in->lines)
        if (value_field(l, tag, field)) return &l;
    return nullptr;
}

// List-directed items of a field: separators are blanks and commas, a slash ends the
// list; an item r*c stands for r copies of c; a quoted item keeps its blanks.
std::vector<std::string> list_items(const std::string &f) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < f.size()) {
        while (i < f.size() && (f[i] == ' ' || f[i] == '\t')) ++i;
        if (i >= f.size() || f[i] == '/') break;
        if (f[i] == ',') { ++i; continue; }
        std::string item;
        if (f[i] == '\'' || f[i] == '"') {
            const char q = f[i++];
            while (i < f.size()) {
                if (f[i] == q) {
                    if (i + 1 < f.size() && f[i + 1] == q) { item += q; i += 2; continue; }
                    ++i;
                    break;
                }
                item += f[i++];
            }
        } else {
            while (i < f.size() && f[i] != ' ' && f[i] != '\t' && f[i] != ',' && f[i] != '/') item += f[i++];
        }
        const size_t star = item.find('*');
        if (star != std::string::npos && star > 0 && std::all_of(item.begin(), item.begin() + star, ::isdigit)) {
            const int r = std::atoi(item.substr(0, star).c_str());
            for (int k = 0; k < r; ++k) out.push_back(item.substr(star + 1));
        } else {
            out.push_back(item);
        }
    }
    return out;
}

bool parse_real(const std::string &t, double *v) {
    if (t.empty()) return false;
    std::string s = t;
    for (auto &c : s)
        if (c == 'd' || c == 'D' || c == 'q' || c == 'Q') c = 'e';
    bool digit = false;
    for (char c : s) {
        if (std::isdigit((unsigned char)c)) digit = true;
        else if (!(c == '+' || c == '-' || c == '.' || c == 'e' || c == 'E')) return false;
    }
    if (!digit) return false;
    char *end = nullptr;
    *v = std::strtod(s.c_str(), &end);
    return end && *end == '\0';
}

bool parse_int(const std::string &t, int *v) {
    if (t.empty()) return false;
    size_t i = (t[0] == '+' || t[0] == '-') ? 1 : 0;
    if (i >= t.size()) return false;
    for (size_t k = i; k < t.size(); ++k)
        if (!std::isdigit((unsigned char)t[k])) return false;
    long long x = std::atoll(t.c_str());
    if (x > 2147483647LL || x < -2147483648LL) return false;
    *v = (int)x;
    return true;
}

}  // namespace

extern "C" {

int mdft_input_read(const char *path, mdft_input **out) {
    if (!path || !out) { set_error("null argument"); return MDFT_E_ARG; }
    *out = nullptr;
    std::ifstream f(path);
    if (!f) { set_error("cannot open input file %s", path); return MDFT_E_IO; }
    mdft_input *in = new mdft_input;
    std::string raw;
    while (std::getline(f, raw)) {
        if (!raw.empty() && raw.back() == '\r') raw.pop_back();
        std::string rec = raw.substr(0, std::min(raw.size(), kRec));  // read(11,'(a)') into character(100)
        rec = adjustl_trim(rec);
        const size_t h = rec.find('#');
        if (h != std::string::npos) rec.resize(h);
        rec = adjustl_trim(rec);
        if (!rec.empty()) in->lines.push_back(rec);
    }
    *out = in;
    return MDFT_OK;
}

int mdft_input_free(mdft_input *in) {
    delete in;
    return MDFT_OK;
}

int mdft_input_nlines(const mdft_input *in, int *n) {
    if (!in || !n) { set_error("null argument"); return MDFT_E_ARG; }
    *n = (int)in->lines.size();
    return MDFT_OK;
}

int mdft_input_line(const mdft_input *in, int i, char *buf, int buflen) {
    if (!in || !buf || buflen <= 0) { set_error("null argument"); return MDFT_E_ARG; }
    if (i < 0 || i >= (int)in->lines.size()) { set_error("line %d out of range", i); return MDFT_E_ARG; }
    std::snprintf(buf, (size_t)buflen, "%s", in->lines[i].c_str());
    return MDFT_OK;
}

int mdft_input_get_dp(const mdft_input *in, const char *tag, int n, double *out, int *found) {
    if (!in || !tag || !out || n < 1 || n > 3) { set_error("null or invalid argument"); return MDFT_E_ARG; }
    std::string field;
    const bool hit = find_tag(in, tag, &field) != nullptr;
    if (found) *found = hit ? 1 : 0;
    if (!hit) return MDFT_OK;
    const auto items = list_items(field);
    if ((int)items.size() < n) { set_error("tag %s: %d value(s) expected in '%s'", tag, n, field.c_str()); return MDFT_E_IO; }
    for (int k = 0; k < n; ++k)
        if (!parse_real(items[k], &out[k])) { set_error("tag %s: '%s' is not a real", tag, items[k].c_str()); return MDFT_E_IO; }
    return MDFT_OK;
}

int mdft_input_get_int(const mdft_input *in, const char *tag, int n, int *out, int *found) {
    if (!in || !tag || !out || n < 1 || n > 3) { set_error("null or invalid argument"); return MDFT_E_ARG; }
    std::string field;
    const bool hit = find_tag(in, tag, &field) != nullptr;
    if (found) *found = hit ? 1 : 0;
    if (!hit) return MDFT_OK;
    const auto items = list_items(field);
    if ((int)items.size() < n) { set_error("tag %s: %d value(s) expected in '%s'", tag, n, field.c_str()); return MDFT_E_IO; }
    for (int k = 0; k < n; ++k)
        if (!parse_int(items[k], &out[k])) { set_error("tag %s: '%s' is not an integer", tag, items[k].c_str()); return MDFT_E_IO; }
    return MDFT_OK;
}

int mdft_input_get_log(const mdft_input *in, const char *tag, int *out, int *found) {
    if (!in || !tag || !out) { set_error("null argument"); return MDFT_E_ARG; }
    std::string field;
    const bool hit = find_tag(in, tag, &field) != nullptr;
    if (found) *found = hit ? 1 : 0;
    if (!hit) return MDFT_OK;
    const auto items = list_items(field);
    const char c = items.empty() || items[0].empty() ? ' ' : items[0][0];
    if (c == 'T' || c == 't') *out = 1;
    else if (c == 'F' || c == 'f') *out = 0;
    else { set_error("tag %s: '%s' is not a logical (T or F)", tag, field.c_str()); return MDFT_E_IO; }
    return MDFT_OK;
}

int mdft_input_get_char(const mdft_input *in, const char *tag, char *out, int outlen, int *found) {
    if (!in || !tag || !out || outlen <= 0) { set_error("null argument"); return MDFT_E_ARG; }
    std::string field;
    const bool hit = find_tag(in, tag, &field) != nullptr;
    if (found) *found = hit ? 1 : 0;
    if (!hit) return MDFT_OK;
    const auto items = list_items(field);
    if (items.empty() || items[0].empty()) { set_error("tag %s: nothing after '='", tag); return MDFT_E_IO; }
    std::string v = items[0].substr(0, 50);  // character(50)
    std::snprintf(out, (size_t)outlen, "%s", v.c_str());
    return MDFT_OK;
}

int mdft_desc_from_input(const mdft_input *in, const char *ck_path, double n0, int precision, int device, mdft_desc *out) {
    if (!in || !out) { set_error("null argument"); return MDFT_E_ARG; }
    int rc;
    int mrso = 2, mmax = 0;
    double L[3] = {128.0, 128.0, 128.0}, T = 300.0;
    if ((rc = mdft_input_get_int(in, "molrotsymorder", 1, &mrso, nullptr))) return rc;   // module_grid.f90:62
    if ((rc = mdft_input_get_dp(in, "boxlen", 3, L, nullptr))) return rc;               // :63
    int nod[3];
    for (int d = 0; d < 3; ++d) nod[d] = (int)std::lround(L[d] / 0.3);                  // :74 default nint(L/0.3)
    if ((rc = mdft_input_get_int(in, "boxnod", 3, nod, nullptr))) return rc;
    if ((rc = mdft_input_get_int(in, "mmax", 1, &mmax, nullptr))) return rc;            // :95
    if ((rc = mdft_input_get_dp(in, "temperature", 1, &T, nullptr))) return rc;        // module_thermo.f90:25
    if (mrso <= 0 || mmax < 0 || !(T > 0) || L[0] <= 0 || L[1] <= 0 || L[2] <= 0 || nod[0] <= 0 || nod[1] <= 0 || nod[2] <= 0) {
        set_error("dft.in: molrotsymorder, boxlen, boxnod and temperature must be > 0, mmax >= 0");
        return MDFT_E_ARG;
    }
    *out = mdft_desc{nod[0], nod[1], nod[2], L[0], L[1], L[2], mmax, mrso, T, n0, ck_path, precision, device};
    return MDFT_OK;
}

int mdft_read_solute(const char *path, double charge_scale, int cap, int *nsite, double *q, double *sig, double *eps, double *xyz,
                     int *Z) {
    if (!path || !nsite) { set_error("null argument"); return MDFT_E_ARG; }
    std::ifstream f(path);
    if (!f) { set_error("solute file %s cannot be opened", path); return MDFT_E_IO; }
    std::string line;
    if (!std::getline(f, line)) { set_error("%s: empty", path); return MDFT_E_IO; }  // comment line
    int n = -1;
    // the count is the first item of the next line(s) (list-directed read skips blank lines)
    while (std::getline(f, line)) {
        const auto it = list_items(line);
        if (it.empty()) continue;
        if (!parse_int(it[0], &n) || n < 0) { set_error("%s: bad site count '%s'", path, it[0].c_str()); return MDFT_E_IO; }
        break;
    }
    if (n < 0) { set_error("%s: no site count", path); return MDFT_E_IO; }
    *nsite = n;
    if (!q) return MDFT_OK;  // size query
    if (n > cap || !sig || !eps || !xyz) { set_error("%s: %d sites, room for %d", path, n, cap); return MDFT_E_ARG; }
    if (!std::getline(f, line)) { set_error("%s: missing comment line before the sites", path); return MDFT_E_IO; }
    std::vector<std::string> items;
    int s = 0;
    // list-directed READ of 8 items per site: items may continue onto the next line
    while (s < n) {
        while ((int)items.size() < 8) {
            if (!std::getline(f, line)) { set_error("%s: site %d incomplete", path, s + 1); return MDFT_E_IO; }
            const auto it = list_items(line);
            items.insert(items.end(), it.begin(), it.end());
        }
        int idx, z;
        double v[6];
        if (!parse_int(items[0], &idx)) { set_error("%s: site %d: bad index '%s'", path, s + 1, items[0].c_str()); return MDFT_E_IO; }
        for (int k = 0; k < 6; ++k)
            if (!parse_real(items[1 + k], &v[k])) { set_error("%s: site %d: '%s' is not a real", path, s + 1, items[1 + k].c_str()); return MDFT_E_IO; }
        if (!parse_int(items[7], &z)) { set_error("%s: site %d: bad atomic number '%s'", path, s + 1, items[7].c_str()); return MDFT_E_IO; }
        q[s] = v[0] * charge_scale;  // solute_charges_scale_factor, module_solute.f90:52
        sig[s] = v[1];
        eps[s] = v[2];
        xyz[3 * s] = v[3];
        xyz[3 * s + 1] = v[4];
        xyz[3 * s + 2] = v[5];
        if (Z) Z[s] = z;
        items.clear();  // a list-directed READ statement consumes the rest of its last record
        ++s;
    }
    return MDFT_OK;
}

int mdft_center_solute(int nsite, double *xyz, const double *box, int translate) {
    if (nsite < 0 || (nsite > 0 && !xyz) || !box) { set_error("null or invalid argument"); return MDFT_E_ARG; }
    if (translate && nsite > 0) {
        for (int d = 0; d < 3; ++d) {
            double mean = 0.0;
            for (int s = 0; s < nsite; ++s) mean += xyz[3 * s + d];
            mean /= (double)nsite;
            const double shift = box[d] / 2.0;
            for (int s = 0; s < nsite; ++s) xyz[3 * s + d] = xyz[3 * s + d] + shift - mean;
        }
    }
    for (int s = 0; s < nsite; ++s)
        for (int d = 0; d < 3; ++d) {
            // Fortran MODULO: result has the sign of the box length
            double r = std::fmod(xyz[3 * s + d], box[d]);
            if (r != 0.0 && ((r < 0.0) != (box[d] < 0.0))) r += box[d];
            xyz[3 * s + d] = r;
        }
    return MDFT_OK;
}

}  // extern "C"
