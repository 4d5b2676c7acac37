// host_io.cpp -- readers of the reference's input files behind the C ABI.
//   boundary.dat / boundary<N>.dat  read_boundary (airfoil.f90:191-242), format (2f14.8)
//   motion_params.dat               load_motion_table (mode.f90:68-142), list-directed rows
#include <algorithm>
#include <cerrno>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "lbm_internal.h"

namespace {

bool parse_double(const std::string &tok, double &out)
{
    std::string t = tok;
    for (char &c : t)
        if (c == 'd' || c == 'D') c = 'e';   // Fortran exponent letter
    char *end = nullptr;
    errno = 0;
    out = strtod(t.c_str(), &end);
    return end && *end == '\0' && errno == 0 && !t.empty();
}

std::vector<std::string> split(const std::string &line)
{
    std::vector<std::string> out;
    std::string cur;
    for (char c : line) {
        if (c == ' ' || c == '\t' || c == ',' || c == '\r' || c == '\n') {
            if (!cur.empty()) out.push_back(cur), cur.clear();
        } else {
            cur += c;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

bool blank(const std::string &s)
{
    for (char c : s)
        if (c != ' ' && c != '\t' && c != '\r') return false;
    return true;
}

// one (2f14.8) record: two 14-character fields; a record written with other
// spacing is accepted when it splits into two numbers
bool read_pair(const std::string &line, double &x, double &y)
{
    if (line.size() >= 28) {
        std::string a = line.substr(0, 14), b = line.substr(14, 14);
        auto trim = [](std::string s) {
            size_t p = s.find_first_not_of(" \t"), q = s.find_last_not_of(" \t\r");
            return p == std::string::npos ? std::string() : s.substr(p, q - p + 1);
        };
        if (parse_double(trim(a), x) && parse_double(trim(b), y)) return true;
    }
    auto t = split(line);
    return t.size() >= 2 && parse_double(t[0], x) && parse_double(t[1], y);
}

// reads npts (2f14.8) records; returns an LBM status and a message
int parse_boundary(const std::string &path, int npts, std::vector<double> &x, std::vector<double> &y,
                   std::string &msg)
{
    std::ifstream in(path);
    if (!in) {
        msg = "cannot open boundary file: " + path;                    // airfoil.f90:225-228
        return LBM_ERR_IO;
    }
    x.clear();
    y.clear();
    std::string line;
    while ((int)x.size() < npts && std::getline(in, line)) {
        double a, b;
        if (!read_pair(line, a, b)) {
            msg = "malformed boundary file: " + path;                   // airfoil.f90:231-234
            return LBM_ERR_IO;
        }
        x.push_back(a);
        y.push_back(b);
    }
    if ((int)x.size() < npts) {
        msg = "boundary file has fewer than points_per_wing records: " + path;
        return LBM_ERR_IO;
    }
    return LBM_OK;
}

// reads the non-blank list-directed rows of a motion file (row-major)
int parse_motion(const std::string &path, int cols, std::vector<std::vector<double>> &rows, std::string &msg)
{
    std::ifstream in(path);
    if (!in) {
        msg = "cannot open motion file: " + path;                      // mode.f90:82-86
        return LBM_ERR_IO;
    }
    rows.clear();
    std::string line;
    while (std::getline(in, line)) {
        if (blank(line)) continue;                                   // mode.f90:91
        auto t = split(line);
        if ((int)t.size() < cols) {
            msg = "motion file format error: each row needs 1+9*wing_count values";   // mode.f90:94-97
            return LBM_ERR_IO;
        }
        std::vector<double> r(cols);
        for (int c = 0; c < cols; ++c)
            if (!parse_double(t[c], r[c])) {
                msg = "motion file format error: not a number";
                return LBM_ERR_IO;
            }
        rows.push_back(r);
    }
    if (rows.empty()) {
        msg = "motion file is empty";                                 // mode.f90:101-104
        return LBM_ERR_IO;
    }
    return LBM_OK;
}

}  // namespace

extern "C" int lbm_parse_boundary_file(const char *path, int npts, double *x, double *y)
{
    if (!path || npts < 1 || !x || !y) return LBM_ERR_ARG;
    std::vector<double> vx, vy;
    std::string msg;
    int rc = parse_boundary(path, npts, vx, vy, msg);
    if (rc) return rc;
    std::copy(vx.begin(), vx.end(), x);
    std::copy(vy.begin(), vy.end(), y);
    return LBM_OK;
}

extern "C" int lbm_parse_motion_file(const char *path, int cols, double *table, int max_rows, int *rows)
{
    if (!path || cols < 1 || !rows) return LBM_ERR_ARG;
    std::vector<std::vector<double>> r;
    std::string msg;
    int rc = parse_motion(path, cols, r, msg);
    if (rc) return rc;
    *rows = (int)r.size();
    if (!table) return LBM_OK;
    if ((int)r.size() > max_rows) return LBM_ERR_ARG;
    for (int i = 0; i < (int)r.size(); ++i)
        for (int c = 0; c < cols; ++c) table[(size_t)c * max_rows + i] = r[i][c];
    return LBM_OK;
}

extern "C" int lbm_read_boundary(lbm_t *h, const char *dir)
{
    if (!h) return LBM_ERR_ARG;
    std::string d = dir ? dir : "";
    if (!d.empty() && d.back() != '/') d += '/';
    for (int w = 1; w <= h->nwing; ++w) {
        const std::string name = w == 1 ? "boundary.dat" : "boundary" + std::to_string(w - 1) + ".dat";  // airfoil.f90:199-204
        std::vector<double> x, y;
        int rc = parse_boundary(d + name, h->ppw, x, y, h->err);
        if (rc) return rc;
        rc = lbm_set_boundary(h, w, x.data(), y.data(), h->ppw);
        if (rc) return rc;
    }
    return LBM_OK;
}

extern "C" int lbm_load_motion_table(lbm_t *h, const char *path)
{
    if (!h) return LBM_ERR_ARG;
    const int cols = 1 + 9 * h->nwing;
    std::vector<std::vector<double>> rows;
    int rc = parse_motion(path ? path : "motion_params.dat", cols, rows, h->err);
    if (rc) return rc;
    const int nr = (int)rows.size();
    std::vector<double> tab((size_t)nr * cols);
    for (int r = 0; r < nr; ++r)
        for (int c = 0; c < cols; ++c) tab[(size_t)c * nr + r] = rows[r][c];
    return lbm_set_motion_table(h, tab.data(), nr, cols);
}
