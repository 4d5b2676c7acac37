// output_io.cu -- the reference's output and restart files behind the C ABI.
//   F<n>.dat     output (solution.f90:129-238): Tecplot ASCII; a field zone
//                sampled every stride-th node (X, Y, U/UU, V/UU, pressure
//                rho/3, vorticity, body, dvordt) and an FE-triangle zone of
//                the airfoil contour with one centre node per wing.
//   checkpoint   saveflowfield / readflowfield (solution.f90:1604-1839): the
//                same two-file scheme (the file and its "_copy"; the reader
//                falls back to the copy when the file is missing, short or
//                corrupt), holding this library's exact device state so that
//                a restart continues bit for bit.
//   saved_flow_feild.dat   the same routines in the reference's own byte
//                layout (nvfortran form='binary'), so that a run can move
//                between the reference and this library in either direction.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "lbm_internal.h"

namespace {

int io_err(lbm_handle *h, int code, const std::string &msg)
{
    if (h) h->err = msg;
    return code;
}

// Fortran Ew.d editing: 0.d1..dd E+xx (E dropped for a 3-digit exponent),
// right-justified in w characters, asterisks when it does not fit.
int fmt_e(char *out, double x, int w, int d)
{
    char tmp[64];
    int n;
    if (std::isnan(x)) {
        n = snprintf(tmp, sizeof tmp, "NaN");
    } else if (std::isinf(x)) {
        n = snprintf(tmp, sizeof tmp, x < 0 ? "-Infinity" : "Infinity");
    } else if (x == 0.0) {
        std::string z = std::string(std::signbit(x) ? "-" : "") + "0." + std::string(d, '0') + "E+00";
        n = snprintf(tmp, sizeof tmp, "%s", z.c_str());
    } else {
        char sci[64];
        snprintf(sci, sizeof sci, "%.*e", d - 1, std::fabs(x));   // d significant digits, rounded
        // sci = D.DDDDDDDe[+-]XX
        std::string digits;
        digits += sci[0];
        const char *p = sci + 1;
        if (*p == '.') ++p;
        while (*p && *p != 'e') digits += *p++;
        const int ex = atoi(p + 1) + 1;   // 0.DDDD x 10^ex
        const char sign = ex < 0 ? '-' : '+';
        const int ax = std::abs(ex);
        if (ax <= 99)
            n = snprintf(tmp, sizeof tmp, "%s0.%sE%c%02d", x < 0 ? "-" : "", digits.c_str(), sign, ax);
        else
            n = snprintf(tmp, sizeof tmp, "%s0.%s%c%03d", x < 0 ? "-" : "", digits.c_str(), sign, ax);
    }
    if (n > w) {
        memset(out, '*', w);
    } else {
        memset(out, ' ', w - n);
        memcpy(out + (w - n), tmp, n);
    }
    return w;
}

// Fortran Fw.d editing, asterisks when it does not fit
int fmt_f(char *out, double x, int w, int d)
{
    char tmp[128];
    const int n = snprintf(tmp, sizeof tmp, "%*.*f", w, d, x);
    if (n > w)
        memset(out, '*', w);
    else
        memcpy(out, tmp, w);
    return w;
}

struct FieldGrid {
    int nx, ny, sx, sy;
    double ox, oy, scale, uu;
    const double *rho, *u, *v;
};

// one line of the field zone for node (i, j), 0-based: format (25e16.8)
// of X, Y, U/UU, V/UU, rho/3, vorticity (solution.f90:194-210), body, dvordt
int field_line(const FieldGrid &g, int i, int j, char *out)
{
    const long long nx = g.nx;
    auto U = [&](int a, int b) { return g.u[(size_t)b * nx + a]; };
    auto V = [&](int a, int b) { return g.v[(size_t)b * nx + a]; };
    const double h = g.uu * g.scale;
    double dvx, duy;
    if (i == g.nx - 1)
        dvx = (1.5 * V(i, j) - 2.0 * V(i - 1, j) + 0.5 * V(i - 2, j)) / h;
    else if (i == 0)
        dvx = (-1.5 * V(i, j) + 2.0 * V(i + 1, j) - 0.5 * V(i + 2, j)) / h;
    else
        dvx = (V(i + 1, j) - V(i - 1, j)) / (g.uu * 2.0 * g.scale);
    if (j == g.ny - 1)
        duy = (1.5 * U(i, j) - 2.0 * U(i, j - 1) + 0.5 * U(i, j - 2)) / h;
    else if (j == 0)
        duy = (-1.5 * U(i, j) + 2.0 * U(i, j + 1) - 0.5 * U(i, j + 2)) / h;
    else
        duy = (U(i, j + 1) - U(i, j - 1)) / (g.uu * 2.0 * g.scale);
    const double vals[8] = {g.ox + (double)i * g.scale, g.oy + (double)j * g.scale, U(i, j) / g.uu, V(i, j) / g.uu,
                            g.rho[(size_t)j * nx + i] / 3.0, dvx - duy, 0.0, 0.0};
    int k = 0;
    for (int c = 0; c < 8; ++c) k += fmt_e(out + k, vals[c], 16, 8);
    out[k++] = '\n';
    return k;
}

// "ZONE ..." header items in list-directed style: integers in 12 columns,
// reals with 17 significant digits
std::string ld_int(long long v)
{
    char b[32];
    snprintf(b, sizeof b, "%12lld", v);
    return b;
}
std::string ld_real(double v)
{
    char b[48];
    snprintf(b, sizeof b, "%25.16E", v);
    return b;
}

bool write_all(FILE *f, const void *p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }

// the field zone written by threads into per-chunk buffers, in row order
bool write_field_zone(FILE *f, const FieldGrid &g)
{
    const int ox = (g.nx - 1) / g.sx + 1, oy = (g.ny - 1) / g.sy + 1;
    const int line = 8 * 16 + 1;
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt ? std::min(nt, 32u) : 4u;
    const int rows_per_chunk = std::max(1, (int)(4u << 20) / (line * ox));   // ~4 MB of text per chunk
    for (int r0 = 0; r0 < oy; r0 += rows_per_chunk * (int)nt) {
        std::vector<std::string> buf(nt);
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) {
            const int a = r0 + (int)t * rows_per_chunk, b = std::min(oy, a + rows_per_chunk);
            if (a >= b) break;
            th.emplace_back([&, t, a, b]() {
                std::string &s = buf[t];
                s.resize((size_t)(b - a) * ox * line);
                char *p = &s[0];
                for (int jr = a; jr < b; ++jr)
                    for (int ir = 0; ir < ox; ++ir) p += field_line(g, ir * g.sx, jr * g.sy, p);
            });
        }
        for (auto &x : th) x.join();
        for (unsigned t = 0; t < th.size(); ++t)
            if (!write_all(f, buf[t].data(), buf[t].size())) return false;
    }
    return true;
}

// g<n>.dat of the reference's output_gforce (solution.f90:240-267): one line
// of (25e25.17) per position of its loop, which runs i over 1..Ny (outer)
// and j over 1..Nx and writes ox + (i-1) scale, oy + (j-1) scale,
// gforce(i,j,1), gforce(i,j,2), as written. gforce is an (Nx,Ny) array;
// positions the loop reaches outside it (j > Ny when Nx > Ny) and null
// arrays write 0, the value gforce holds on the live path (move_boundary
// zeroes it at the support nodes, airfoil.f90:280-281, and no live routine
// writes it).
struct GforceGrid {
    int nx, ny;
    double ox, oy, scale;
    const double *gx, *gy;   // (nx, ny), x fastest; nullable
};

int gforce_line(const GforceGrid &g, int i, int j, char *out)   // loop position, 0-based
{
    double fx = 0.0, fy = 0.0;
    if (i < g.nx && j < g.ny) {
        const size_t q = (size_t)j * g.nx + i;
        if (g.gx) fx = g.gx[q];
        if (g.gy) fy = g.gy[q];
    }
    const double vals[4] = {g.ox + (double)i * g.scale, g.oy + (double)j * g.scale, fx, fy};
    int k = 0;
    for (int c = 0; c < 4; ++c) k += fmt_e(out + k, vals[c], 25, 17);
    out[k++] = '\n';
    return k;
}

// the rows of the loop (i) written by threads into per-chunk buffers, in order
bool write_gforce_zone(FILE *f, const GforceGrid &g)
{
    const int line = 4 * 25 + 1;
    unsigned nt = std::thread::hardware_concurrency();
    nt = nt ? std::min(nt, 32u) : 4u;
    const int rows_per_chunk = std::max(1, (int)(4u << 20) / (line * g.nx));   // ~4 MB of text per chunk
    for (int r0 = 0; r0 < g.ny; r0 += rows_per_chunk * (int)nt) {
        std::vector<std::string> buf(nt);
        std::vector<std::thread> th;
        for (unsigned t = 0; t < nt; ++t) {
            const int a = r0 + (int)t * rows_per_chunk, b = std::min(g.ny, a + rows_per_chunk);
            if (a >= b) break;
            th.emplace_back([&, t, a, b]() {
                std::string &s = buf[t];
                s.resize((size_t)(b - a) * g.nx * line);
                char *p = &s[0];
                for (int i = a; i < b; ++i)
                    for (int j = 0; j < g.nx; ++j) p += gforce_line(g, i, j, p);
            });
        }
        for (auto &x : th) x.join();
        for (unsigned t = 0; t < th.size(); ++t)
            if (!write_all(f, buf[t].data(), buf[t].size())) return false;
    }
    return true;
}

// contour points xb1, yb1 (airfoil.f90:255-266) of step `s` (1-based step
// index of the motion table row the step used)
void contour_points(const lbm_handle *h, int s, std::vector<double> &x, std::vector<double> &y)
{
    const int row = std::max(1, std::min(s, h->msteps)) - 1;
    const double *r = h->mstep_host.data() + (size_t)row * h->mcols;
    x.assign(h->npts, 0.0);
    y.assign(h->npts, 0.0);
    for (int w = 0; w < h->nwing; ++w) {
        const double angle = r[1 + 9 * w], sa = r[4 + 9 * w], sb = r[7 + 9 * w];
        const double ca = cos(angle), sn = sin(angle);
        for (int p = 0; p < h->ppw; ++p) {
            const int q = w * h->ppw + p;
            x[q] = ca * h->hx0[q] + sn * h->hy0[q] + sa + h->p.xc;
            y[q] = -sn * h->hx0[q] + ca * h->hy0[q] + sb + h->p.yc;
        }
    }
}

int write_tecplot(const char *path, int cycle, const FieldGrid &g, double soltime, int nwing, int ppw,
                  const double *xb1, const double *yb1, std::string &msg)
{
    FILE *f = fopen(path, "wb");
    if (!f) {
        msg = std::string("cannot open ") + path;
        return LBM_ERR_IO;
    }
    const int ox = (g.nx - 1) / g.sx + 1, oy = (g.ny - 1) / g.sy + 1;
    std::string head = "VARIABLES = \"X\" \"Y\" \"U\" \"V\" \"Presure\" \"Vorticity\" \"body\" \"dvordt\" \n";
    head += " ZONE T=\"Flow feild\", I=" + ld_int(ox) + " ,J=" + ld_int(oy) + " ,SOLUTIONTIME=" + ld_real(soltime) + "\n";
    bool ok = write_all(f, head.data(), head.size()) && write_field_zone(f, g);
    if (ok && nwing > 0) {
        const int bpoint = nwing * ppw, bseg = nwing * (ppw - 1);
        std::string z = " ZONE T=\"airfoil\", NODES=" + ld_int(bpoint + nwing) + " ELEMENTS,=" + ld_int(bseg) +
                        ", DATAPACKING=POINT, ZONETYPE=FETRIANGLE,SOLUTIONTIME=" + ld_real(soltime) + "\n";
        char line[256];
        auto point = [&](double x, double y) {   // (8f14.8)
            const double v[8] = {x, y, 255.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            int k = 0;
            for (int c = 0; c < 8; ++c) k += fmt_f(line + k, v[c], 14, 8);
            line[k++] = '\n';
            z.append(line, k);
        };
        for (int q = 0; q < bpoint; ++q) point(xb1[q], yb1[q]);
        for (int w = 0; w < nwing; ++w) {   // centre node: between the first point and the one halfway round
            const int j = w * ppw, k = j + (ppw - 1) / 2;
            point(0.5 * (xb1[j] + xb1[k]), 0.5 * (yb1[j] + yb1[k]));
        }
        for (int w = 0; w < nwing; ++w)   // (3I5.3), 1-based node numbers
            for (int k = w * ppw + 1; k <= w * ppw + ppw - 1; ++k) {
                const int n = snprintf(line, sizeof line, "%5.3d%5.3d%5.3d\n", k, k + 1, bpoint + w + 1);
                z.append(line, n);
            }
        ok = write_all(f, z.data(), z.size());
    }
    ok = (fclose(f) == 0) && ok;
    if (!ok) msg = std::string("write failed: ") + path;
    (void)cycle;
    return ok ? LBM_OK : LBM_ERR_IO;
}

// ---- checkpoint ---------------------------------------------------------

const char kMagic[16] = {'L', 'B', 'M', 'B', '2', '0', '0', ' ', 'C', 'K', 'P', 'T', ' ', 'v', '1', '\0'};

struct CkptHeader {
    int32_t version, nx, ny, pitch, prec, nwing, ppw, cur;
    int64_t n, steps_done, fields_step[2];
    int32_t fields_slot, pad;
    int64_t pop_bytes, edge_bytes, field_bytes;
};

uint64_t fnv1a(uint64_t hsh, const void *p, size_t n)
{
    const unsigned char *b = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) {
        hsh ^= b[i];
        hsh *= 1099511628211ull;
    }
    return hsh;
}

std::string copy_path(const std::string &path)
{
    const size_t slash = path.find_last_of('/');
    const size_t dot = path.find_last_of('.');
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return path + "_copy";
    return path.substr(0, dot) + "_copy" + path.substr(dot);
}

size_t edge_bytes(const lbm_handle *h)
{
    const size_t cs = h->prec == LBM_PREC_FP64 ? 8 : 4;
    return cs * (6 * (size_t)h->ny + 36);
}

size_t field_bytes(const lbm_handle *h)
{
    const size_t cs = h->prec == LBM_PREC_FP64 ? 8 : 4;
    return 3 * cs * (size_t)h->nx * h->ny;
}

// the FP64 edge f0 the boundary values were built from (lbm_handle::edge_f0)
size_t ef0_bytes(const lbm_handle *h) { return sizeof(double) * 9 * (2 * (size_t)h->nx + 2 * (size_t)h->ny); }

// the whole state in host memory (header, populations, edge values, fields x2,
// edge f0)
int gather_state(lbm_handle *h, CkptHeader &hd, std::vector<unsigned char> &blob)
{
    hd = CkptHeader{};
    hd.version = 2;
    hd.nx = h->nx; hd.ny = h->ny; hd.pitch = h->pitch; hd.prec = h->prec;
    hd.nwing = h->nwing; hd.ppw = h->ppw; hd.cur = 0;
    hd.n = h->n; hd.steps_done = h->steps_done;
    hd.fields_step[0] = h->fields_step[0]; hd.fields_step[1] = h->fields_step[1];
    hd.fields_slot = h->fields_slot;
    hd.pop_bytes = (int64_t)(h->elem * 9 * (size_t)h->plane);
    hd.edge_bytes = (int64_t)edge_bytes(h);
    hd.field_bytes = (int64_t)field_bytes(h);
    blob.resize((size_t)(hd.pop_bytes + hd.edge_bytes + 2 * hd.field_bytes) + ef0_bytes(h));
    unsigned char *p = blob.data();
    cudaError_t e = cudaMemcpyAsync(p, h->fbuf[h->cur], hd.pop_bytes, cudaMemcpyDeviceToHost, h->stream);
    p += hd.pop_bytes;
    if (e == cudaSuccess) e = cudaMemcpyAsync(p, h->edge_c, hd.edge_bytes, cudaMemcpyDeviceToHost, h->stream);
    p += hd.edge_bytes;
    for (int s = 0; s < 2 && e == cudaSuccess; ++s, p += hd.field_bytes)
        e = cudaMemcpyAsync(p, h->d_fields[s], hd.field_bytes, cudaMemcpyDeviceToHost, h->stream);
    memcpy(p, h->edge_f0.data(), ef0_bytes(h));
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return io_err(h, LBM_ERR_CUDA, std::string("checkpoint: ") + cudaGetErrorString(e));
    return LBM_OK;
}

int write_ckpt_file(const std::string &path, const CkptHeader &hd, const std::vector<unsigned char> &blob)
{
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return LBM_ERR_IO;
    uint64_t sum = fnv1a(1469598103934665603ull, &hd, sizeof hd);
    sum = fnv1a(sum, blob.data(), blob.size());
    bool ok = write_all(f, kMagic, sizeof kMagic) && write_all(f, &hd, sizeof hd) &&
              write_all(f, blob.data(), blob.size()) && write_all(f, &sum, sizeof sum);
    ok = (fclose(f) == 0) && ok;
    return ok ? LBM_OK : LBM_ERR_IO;
}

// reads and checks one checkpoint file against the handle; "" on success
std::string read_ckpt_file(const lbm_handle *h, const std::string &path, CkptHeader &hd, std::vector<unsigned char> &blob)
{
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return "cannot open " + path;
    char magic[16];
    std::string why;
    if (fread(magic, 1, 16, f) != 16 || memcmp(magic, kMagic, 16) != 0) why = "not a checkpoint of this library";
    else if (fread(&hd, 1, sizeof hd, f) != sizeof hd) why = "short header";
    else if (hd.version != 2) why = "unknown checkpoint version";
    else if (hd.nx != h->nx || hd.ny != h->ny || hd.pitch != h->pitch || hd.prec != h->prec || hd.nwing != h->nwing ||
             hd.ppw != h->ppw)
        why = "grid, storage precision or wings differ from this case";
    else if (hd.pop_bytes != (int64_t)(h->elem * 9 * (size_t)h->plane) || hd.edge_bytes != (int64_t)edge_bytes(h) ||
             hd.field_bytes != (int64_t)field_bytes(h))
        why = "section sizes differ from this case";
    if (why.empty()) {
        blob.resize((size_t)(hd.pop_bytes + hd.edge_bytes + 2 * hd.field_bytes) + ef0_bytes(h));
        uint64_t sum = 0;
        if (fread(blob.data(), 1, blob.size(), f) != blob.size() || fread(&sum, 1, sizeof sum, f) != sizeof sum)
            why = "short file";
        else if (sum != fnv1a(fnv1a(1469598103934665603ull, &hd, sizeof hd), blob.data(), blob.size()))
            why = "checksum mismatch";
    }
    fclose(f);
    return why.empty() ? "" : path + ": " + why;
}

// ---- restart file in the reference's layout ------------------------------
// saveflowfield (solution.f90:1646-1672) opens the file form='binary':
// unformatted with no record markers, native byte order, so the file is the
// items of each WRITE back to back:
//   int32 cycle1, int32 wing_count,
//   11 x wing_count float64: body_rel_a, _a_prev, _v, _v_prev, _s, _s_prev,
//     _pos, _theta_prev, _theta, _temp_theta_prev, _temp_theta,
//   int32 movenum,
//   j = 1..Ny, i = 1..Nx: float64 u(i,j), v(i,j), f(i,j,1:9),
//   j = 2..Ny-1: leftf2(j,:), f0(1,j,:), rightf2(j,:), f0(Nx,j,:),
//   i = 1..Nx:   upf2(i,:), f0(i,Ny,:), downf2(i,:), f0(i,1,:).
// leftf2 .. downf2 are copies of the initial edge populations
// (solution.f90:60-63) that only the multi-block refinement rewrites
// (solution.f90:1300-1360, not called with one mesh), so they equal the edge
// f0 and are written from it; the reader does not use them.

const int kBodyArrays = 11;

size_t flow_file_bytes(int nx, int ny, int nwing)
{
    return 12 + 8 * (size_t)kBodyArrays * nwing + 88 * (size_t)nx * ny + 8 * 36 * ((size_t)(ny - 2) + (size_t)nx);
}

int write_flow_file(const char *path, int nx, int ny, int cycle, int nwing, const double *body, int movenum,
                    const double *u, const double *v, const double *f, const double *ef)
{
    FILE *fp = fopen(path, "wb");
    if (!fp) return LBM_ERR_IO;
    const size_t nn = (size_t)nx * ny;
    const int32_t head[2] = {cycle, nwing};
    std::vector<double> zeros((size_t)kBodyArrays * nwing, 0.0);
    const int32_t mv = movenum;
    bool ok = write_all(fp, head, sizeof head) &&
              write_all(fp, body ? body : zeros.data(), sizeof(double) * kBodyArrays * nwing) &&
              write_all(fp, &mv, sizeof mv);
    std::vector<double> row(11 * (size_t)nx);
    for (int j = 0; j < ny && ok; ++j) {
        for (int i = 0; i < nx; ++i) {
            const size_t q = (size_t)j * nx + i;
            double *o = row.data() + 11 * (size_t)i;
            o[0] = u[q];
            o[1] = v[q];
            for (int k = 0; k < 9; ++k) o[2 + k] = f[k * nn + q];
        }
        ok = write_all(fp, row.data(), sizeof(double) * row.size());
    }
    const double *L = ef, *R = ef + 9 * (size_t)ny, *B = ef + 18 * (size_t)ny, *T = B + 9 * (size_t)nx;
    std::vector<double> edge(36 * (size_t)std::max(nx, ny));
    double *o = edge.data();
    for (int j = 1; j < ny - 1; ++j)
        for (const double *src : {L + 9 * (size_t)j, L + 9 * (size_t)j, R + 9 * (size_t)j, R + 9 * (size_t)j}) {
            memcpy(o, src, 9 * sizeof(double));
            o += 9;
        }
    if (ok) ok = write_all(fp, edge.data(), sizeof(double) * (size_t)(o - edge.data()));
    o = edge.data();
    for (int i = 0; i < nx; ++i)
        for (const double *src : {T + 9 * (size_t)i, T + 9 * (size_t)i, B + 9 * (size_t)i, B + 9 * (size_t)i}) {
            memcpy(o, src, 9 * sizeof(double));
            o += 9;
        }
    if (ok) ok = write_all(fp, edge.data(), sizeof(double) * (size_t)(o - edge.data()));
    ok = (fclose(fp) == 0) && ok;
    return ok ? LBM_OK : LBM_ERR_IO;
}

// reads one file of the layout above. Returns LBM_OK, LBM_ERR_IO for a file
// that is missing, short or of another size (the reader of the reference
// then tries the copy: err=/end= branches, solution.f90:1738-1744), or
// LBM_ERR_STATE for a wing count other than this case's (the reference
// stops, solution.f90:1740); `why` says which.
int read_flow_file(const char *path, int nx, int ny, int nwing, int *cycle, double *body, int *movenum, double *u,
                   double *v, double *f, double *ef, std::string &why)
{
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        why = std::string("cannot open ") + path;
        return LBM_ERR_IO;
    }
    auto fail = [&](int code, const std::string &w) {
        fclose(fp);
        why = std::string(path) + ": " + w;
        return code;
    };
    int32_t head[2];
    if (fread(head, sizeof head, 1, fp) != 1) return fail(LBM_ERR_IO, "short file");
    if (head[1] != nwing) return fail(LBM_ERR_STATE, "wing count " + std::to_string(head[1]) + " in the file, " +
                                                         std::to_string(nwing) + " in this case");
    if (fseek(fp, 0, SEEK_END) != 0) return fail(LBM_ERR_IO, "cannot seek");
    const long long size = ftell(fp);
    const size_t want = flow_file_bytes(nx, ny, nwing);
    if (size < 0 || (size_t)size != want)
        return fail(LBM_ERR_IO, "size " + std::to_string(size) + " bytes, a " + std::to_string(nx) + "x" +
                                    std::to_string(ny) + " grid with " + std::to_string(nwing) + " wings has " +
                                    std::to_string(want));
    if (fseek(fp, 8, SEEK_SET) != 0) return fail(LBM_ERR_IO, "cannot seek");
    std::vector<double> bs((size_t)kBodyArrays * nwing);
    int32_t mv = 0;
    if ((nwing > 0 && fread(bs.data(), sizeof(double), bs.size(), fp) != bs.size()) || fread(&mv, sizeof mv, 1, fp) != 1)
        return fail(LBM_ERR_IO, "short file");
    const size_t nn = (size_t)nx * ny;
    std::vector<double> row(11 * (size_t)nx);
    for (int j = 0; j < ny; ++j) {
        if (fread(row.data(), sizeof(double), row.size(), fp) != row.size()) return fail(LBM_ERR_IO, "short file");
        for (int i = 0; i < nx; ++i) {
            const size_t q = (size_t)j * nx + i;
            const double *x = row.data() + 11 * (size_t)i;
            u[q] = x[0];
            v[q] = x[1];
            for (int k = 0; k < 9; ++k) f[k * nn + q] = x[2 + k];
        }
    }
    double *L = ef, *R = ef + 9 * (size_t)ny, *B = ef + 18 * (size_t)ny, *T = B + 9 * (size_t)nx;
    double rec[36];
    for (int j = 1; j < ny - 1; ++j) {   // leftf2, f0(1,j), rightf2, f0(Nx,j)
        if (fread(rec, sizeof(double), 36, fp) != 36) return fail(LBM_ERR_IO, "short file");
        memcpy(L + 9 * (size_t)j, rec + 9, 9 * sizeof(double));
        memcpy(R + 9 * (size_t)j, rec + 27, 9 * sizeof(double));
    }
    for (int i = 0; i < nx; ++i) {       // upf2, f0(i,Ny), downf2, f0(i,1)
        if (fread(rec, sizeof(double), 36, fp) != 36) return fail(LBM_ERR_IO, "short file");
        memcpy(T + 9 * (size_t)i, rec + 9, 9 * sizeof(double));
        memcpy(B + 9 * (size_t)i, rec + 27, 9 * sizeof(double));
    }
    fclose(fp);
    // the corner nodes of the columns are those of the rows
    memcpy(L, B, 9 * sizeof(double));
    memcpy(L + 9 * (size_t)(ny - 1), T, 9 * sizeof(double));
    memcpy(R, B + 9 * (size_t)(nx - 1), 9 * sizeof(double));
    memcpy(R + 9 * (size_t)(ny - 1), T + 9 * (size_t)(nx - 1), 9 * sizeof(double));
    *cycle = head[0];
    *movenum = mv;
    if (body) std::copy(bs.begin(), bs.end(), body);
    return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_write_flow_field_file(const char *path, int nx, int ny, int cycle, int wing_count, const double *body_state,
                              int movenum, const double *u, const double *v, const double *f, const double *edge_f0)
{
    if (!path || nx < 3 || ny < 3 || wing_count < 0 || !u || !v || !f || !edge_f0) return LBM_ERR_ARG;
    return write_flow_file(path, nx, ny, cycle, wing_count, body_state, movenum, u, v, f, edge_f0);
}

int lbm_read_flow_field_file(const char *path, int nx, int ny, int wing_count, int *cycle, double *body_state,
                             int *movenum, double *u, double *v, double *f, double *edge_f0)
{
    if (!path || nx < 3 || ny < 3 || wing_count < 0 || !cycle || !movenum || !u || !v || !f || !edge_f0)
        return LBM_ERR_ARG;
    std::string why;
    return read_flow_file(path, nx, ny, wing_count, cycle, body_state, movenum, u, v, f, edge_f0, why);
}

int lbm_save_flow_field(lbm_t *h, const char *path, const double *body_state, int movenum)
{
    if (!h || !path) return LBM_ERR_ARG;
    if (!h->inited) return io_err(h, LBM_ERR_STATE, "save_flow_field: not initialised");
    const size_t nn = (size_t)h->nx * h->ny;
    std::vector<double> u(nn), v(nn), f(9 * nn);
    int rc = lbm_get_fields(h, nullptr, u.data(), v.data());
    if (rc) return rc;
    rc = lbm_get_populations(h, f.data());
    if (rc) return rc;
    const std::string p = path, c = copy_path(p);
    for (const std::string &q : {p, c})   // saved_flow_feild.dat and saved_flow_feild_copy.dat
        if (write_flow_file(q.c_str(), h->nx, h->ny, h->n - 1, h->nwing, body_state, movenum, u.data(), v.data(),
                            f.data(), h->edge_f0.data()))
            return io_err(h, LBM_ERR_IO, "save_flow_field: cannot write " + q);
    return LBM_OK;
}

int lbm_read_flow_field(lbm_t *h, const char *path, int *cycle, double *body_state, int *movenum)
{
    if (!h || !path) return LBM_ERR_ARG;
    if (!h->inited) return io_err(h, LBM_ERR_STATE, "read_flow_field: call lbm_init first");
    const size_t nn = (size_t)h->nx * h->ny;
    std::vector<double> u(nn), v(nn), f(9 * nn), ef(9 * (2 * (size_t)h->ny + 2 * (size_t)h->nx));
    std::vector<double> body((size_t)kBodyArrays * h->nwing);
    int cyc = 0, mv = 0;
    const std::string p = path, c = copy_path(p);
    std::string why, why2;
    int rc = read_flow_file(p.c_str(), h->nx, h->ny, h->nwing, &cyc, body.data(), &mv, u.data(), v.data(), f.data(),
                            ef.data(), why);
    if (rc == LBM_ERR_STATE) return io_err(h, rc, "read_flow_field: " + why);
    if (rc) {   // the copy (solution.f90:1768-1802)
        rc = read_flow_file(c.c_str(), h->nx, h->ny, h->nwing, &cyc, body.data(), &mv, u.data(), v.data(), f.data(),
                            ef.data(), why2);
        if (rc) return io_err(h, rc, "read_flow_field: " + why + "; " + why2);
    }
    if (cycle) *cycle = cyc;
    if (movenum) *movenum = mv;
    if (body_state) std::copy(body.begin(), body.end(), body_state);
    // free flight (solve_dynamic_equations, main.f90:103) moves the body and
    // shifts the mesh (move_mesh, main.f90:370-386); the prescribed motion of
    // this library cannot continue such a state
    bool moved = mv != 0;
    for (double b : body) moved = moved || b != 0.0;
    if (moved)
        return io_err(h, LBM_ERR_STATE, "read_flow_field: the file holds rigid-body motion state (free flight or a "
                                        "shifted mesh), which this library does not model");
    if (cyc < 0) return io_err(h, LBM_ERR_IO, "read_flow_field: negative step number in the file");
    return handle_restore(h, f.data(), u.data(), v.data(), ef.data(), cyc);
}

int lbm_write_tecplot_fields(const char *path, int nx, int ny, double ox, double oy, double scale, double uu,
                             double solution_time, int stride_x, int stride_y, const double *rho, const double *u,
                             const double *v, int wing_count, int points_per_wing, const double *xb1, const double *yb1)
{
    if (!path || nx < 3 || ny < 3 || !(scale > 0) || !(uu > 0) || stride_x < 1 || stride_y < 1 || !rho || !u || !v ||
        wing_count < 0 || (wing_count > 0 && (points_per_wing < 3 || !xb1 || !yb1)))
        return LBM_ERR_ARG;
    FieldGrid g{nx, ny, stride_x, stride_y, ox, oy, scale, uu, rho, u, v};
    std::string msg;
    return write_tecplot(path, 0, g, solution_time, wing_count, points_per_wing, xb1, yb1, msg);
}

int lbm_write_gforce(const char *path, int cycle, int nx, int ny, double ox, double oy, double scale,
                     const double *gforce_x, const double *gforce_y)
{
    if (!path || nx < 1 || ny < 1 || !(scale > 0)) return LBM_ERR_ARG;
    FILE *f = fopen(path, "wb");
    if (!f) return LBM_ERR_IO;
    // the two header lines: (a), then list-directed items
    std::string head = "VARIABLES = \"X\" \"Y\" \"gforcex\" \"gforcey\" \n";
    head += " zone,t=\"" + ld_int(cycle) + "\",i=" + ld_int(nx) + ",j=" + ld_int(ny) + "\n";
    GforceGrid g{nx, ny, ox, oy, scale, gforce_x, gforce_y};
    bool ok = write_all(f, head.data(), head.size()) && write_gforce_zone(f, g);
    ok = (fclose(f) == 0) && ok;
    return ok ? LBM_OK : LBM_ERR_IO;
}

int lbm_write_tecplot(lbm_t *h, const char *path, int cycle, int stride_x, int stride_y)
{
    if (!h || !path || stride_x < 1 || stride_y < 1) return LBM_ERR_ARG;
    if (!h->inited) return io_err(h, LBM_ERR_STATE, "write_tecplot: not initialised");
    const size_t nn = (size_t)h->nx * h->ny;
    std::vector<double> rho(nn), u(nn), v(nn);
    int rc = lbm_get_fields(h, rho.data(), u.data(), v.data());
    if (rc) return rc;
    std::vector<double> xb1, yb1;
    if (h->nwing > 0) contour_points(h, h->n - 1, xb1, yb1);
    FieldGrid g{h->nx, h->ny, stride_x, stride_y, h->p.ox, h->p.oy, h->p.scale, h->p.uu,
                rho.data(), u.data(), v.data()};
    std::string msg;
    rc = write_tecplot(path, cycle, g, (double)cycle * h->p.uu * h->p.mesh_max_scale, h->nwing, h->ppw, xb1.data(),
                       yb1.data(), msg);
    return rc ? io_err(h, rc, "write_tecplot: " + msg) : LBM_OK;
}

int lbm_save_checkpoint(lbm_t *h, const char *path)
{
    if (!h || !path) return LBM_ERR_ARG;
    if (!h->inited) return io_err(h, LBM_ERR_STATE, "save_checkpoint: not initialised");
    if (h->fstream) cudaStreamSynchronize(h->fstream);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    CkptHeader hd;
    std::vector<unsigned char> blob;
    int rc = gather_state(h, hd, blob);
    if (rc) return rc;
    const std::string p = path, c = copy_path(p);
    if (write_ckpt_file(p, hd, blob)) return io_err(h, LBM_ERR_IO, "save_checkpoint: cannot write " + p);
    if (write_ckpt_file(c, hd, blob)) return io_err(h, LBM_ERR_IO, "save_checkpoint: cannot write " + c);
    return LBM_OK;
}

int lbm_load_checkpoint(lbm_t *h, const char *path)
{
    if (!h || !path) return LBM_ERR_ARG;
    if (!h->inited) return io_err(h, LBM_ERR_STATE, "load_checkpoint: call lbm_init first");
    CkptHeader hd;
    std::vector<unsigned char> blob;
    const std::string p = path, c = copy_path(p);
    std::string why = read_ckpt_file(h, p, hd, blob);
    if (!why.empty()) {
        const std::string why2 = read_ckpt_file(h, c, hd, blob);   // the copy (readflowfield, solution.f90:1757-1790)
        if (!why2.empty()) return io_err(h, LBM_ERR_IO, "load_checkpoint: " + why + "; " + why2);
    }
    if (h->fstream) cudaStreamSynchronize(h->fstream);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    cudaStreamSynchronize(h->stream);
    const unsigned char *q = blob.data();
    h->cur = 0;
    cudaError_t e = cudaMemcpyAsync(h->fbuf[0], q, hd.pop_bytes, cudaMemcpyHostToDevice, h->stream);
    q += hd.pop_bytes;
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->edge_c, q, hd.edge_bytes, cudaMemcpyHostToDevice, h->stream);
    q += hd.edge_bytes;
    for (int s = 0; s < 2 && e == cudaSuccess; ++s, q += hd.field_bytes)
        e = cudaMemcpyAsync(h->d_fields[s], q, hd.field_bytes, cudaMemcpyHostToDevice, h->stream);
    h->edge_f0.resize(ef0_bytes(h) / sizeof(double));
    memcpy(h->edge_f0.data(), q, ef0_bytes(h));
    if (e == cudaSuccess) e = cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return io_err(h, LBM_ERR_CUDA, std::string("load_checkpoint: ") + cudaGetErrorString(e));
    h->n = (int)hd.n;
    h->steps_done = (int)hd.steps_done;
    h->fields_slot = hd.fields_slot;
    h->fields_step[0] = (int)hd.fields_step[0];
    h->fields_step[1] = (int)hd.fields_step[1];
    // the factorization slots are filled again for the restored step
    h->batch_in_half[0] = h->batch_in_half[1] = -1;
    h->fgroup[0] = h->fgroup[1] = -1;
    return LBM_OK;
}

}  // extern "C"
