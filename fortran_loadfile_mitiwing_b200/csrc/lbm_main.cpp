// lbm_main.cpp -- the reference's driver program (main.f90:159-433) for one
// process and one GPU over the C ABI of lbm_b200.h: set-up (ini_mesh, the
// motion table, init, read_boundary), the optional restart (goon,
// main.f90:320-325), then the time loop (main.f90:351-418) writing
// force.dat and airfoil_motion.dat every step (solution.f90:349-390),
// F<n>.dat on the output steps, saved_flow_feild.dat (+ _copy) on the
// checkpoint steps, and the residual line every 100 steps; the run time at
// the end (main.f90:420-433).
//
// The reference's compile-time PARAMETERs are options here (defaults: the
// reference's own values, lbm_default_params); its output schedule of flag1
// windows (main.f90:396-402) becomes --output-every with an optional window.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"

namespace {

void usage(FILE *f)
{
    fprintf(f,
            "usage: lbm_main [options]\n"
            "  lattice and case (defaults: the reference's PARAMETER values)\n"
            "    --nx N --ny N --wing-count W --points-per-wing P --scale S --ox X --oy Y --uu U --re R\n"
            "    --s1 .. --s9 RATE (s8, s9 <= 0: 1/tau) --xc --yc --xp --yp --mesh-max-scale\n"
            "    --delta peskin4|smooth --precision fp32|fp64|fp16|bf16 --dense-solve\n"
            "  inputs\n"
            "    --boundary-dir DIR     boundary.dat, boundary1.dat, ... (default .)\n"
            "    --motion FILE          motion_params.dat (default ./motion_params.dat)\n"
            "    --restart DIR          continue from DIR/saved_flow_feild.dat (else its _copy);\n"
            "                           rows of DIR/force.dat are not written again\n"
            "  outputs (directory --out, default .)\n"
            "    --steps N              stop after step N (default: the end of the motion table)\n"
            "    --output-every N       F<n>.dat every N steps (0: none; default 0)\n"
            "    --output-window A:B    ... only for A < n <= B\n"
            "    --save-every N         saved_flow_feild.dat every N steps (default 100000; 0: none)\n"
            "    --residual-every N     residual line every N steps (default 100; 0: none)\n"
            "    --chunk N              most steps per lbm_run call (default 500)\n");
}

// Fortran Fw.d editing (asterisks when the value does not fit)
void put_f(std::string &out, double x, int w, int d)
{
    char tmp[128];
    const int n = snprintf(tmp, sizeof tmp, "%*.*f", w, d, x);
    if (n > w || n < 0)
        out.append((size_t)w, '*');
    else
        out.append(tmp, (size_t)n);
}

// one record of format (1000f15.8)
std::string f15_row(const double *v, int n)
{
    std::string s;
    s.reserve((size_t)n * 15 + 1);
    for (int k = 0; k < n; ++k) put_f(s, v[k], 15, 8);
    s += '\n';
    return s;
}

int count_lines(const std::string &path)
{
    FILE *f = fopen(path.c_str(), "r");
    if (!f) return 0;
    int n = 0, c, last = '\n';
    while ((c = fgetc(f)) != EOF) {
        if (c == '\n') ++n;
        last = c;
    }
    if (last != '\n') ++n;
    fclose(f);
    return n;
}

struct Options {
    std::string boundary_dir = ".", motion = "motion_params.dat", out = ".", restart;
    long long steps = -1;
    int output_every = 0, save_every = 100000, residual_every = 100, chunk = 500;
    long long win_a = -1, win_b = -1;
};

bool parse(int argc, char **argv, lbm_params &p, Options &o)
{
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "-h" || a == "--help") {
            usage(stdout);
            exit(0);
        }
        if (a == "--dense-solve") {
            p.flags |= LBM_FLAG_DENSE_SOLVE;
            continue;
        }
        if (i + 1 >= argc) {
            fprintf(stderr, "lbm_main: %s needs a value\n", a.c_str());
            return false;
        }
        const std::string v = argv[++i];
        char *end = nullptr;
        const double x = strtod(v.c_str(), &end);
        const bool num = end && *end == '\0' && !v.empty();
        auto need_num = [&]() {
            if (!num) fprintf(stderr, "lbm_main: %s: not a number: %s\n", a.c_str(), v.c_str());
            return num;
        };
        if (a == "--boundary-dir") o.boundary_dir = v;
        else if (a == "--motion") o.motion = v;
        else if (a == "--out") o.out = v;
        else if (a == "--restart") o.restart = v;
        else if (a == "--delta") {
            if (v == "peskin4") p.delta_kernel = LBM_DELTA_PESKIN4;
            else if (v == "smooth") p.delta_kernel = LBM_DELTA_SMOOTH;
            else { fprintf(stderr, "lbm_main: --delta peskin4|smooth\n"); return false; }
        } else if (a == "--precision") {
            if (v == "fp32") p.precision = LBM_PREC_FP32;
            else if (v == "fp64") p.precision = LBM_PREC_FP64;
            else if (v == "fp16") p.precision = LBM_PREC_FP16;
            else if (v == "bf16") p.precision = LBM_PREC_BF16;
            else { fprintf(stderr, "lbm_main: --precision fp32|fp64|fp16|bf16\n"); return false; }
        } else if (a == "--output-window") {
            long long wa, wb;
            if (sscanf(v.c_str(), "%lld:%lld", &wa, &wb) != 2 || wb < wa) {
                fprintf(stderr, "lbm_main: --output-window A:B with A <= B\n");
                return false;
            }
            o.win_a = wa;
            o.win_b = wb;
        } else {
            if (!need_num()) return false;
            if (a == "--nx") p.nx = (int)x;
            else if (a == "--ny") p.ny = (int)x;
            else if (a == "--wing-count") p.wing_count = (int)x;
            else if (a == "--points-per-wing") p.points_per_wing = (int)x;
            else if (a == "--scale") p.scale = x;
            else if (a == "--ox") p.ox = x;
            else if (a == "--oy") p.oy = x;
            else if (a == "--uu") p.uu = x;
            else if (a == "--re") p.re = x;
            else if (a.size() == 4 && a.compare(0, 3, "--s") == 0 && a[3] >= '1' && a[3] <= '9') p.s[a[3] - '1'] = x;
            else if (a == "--xc") p.xc = x;
            else if (a == "--yc") p.yc = x;
            else if (a == "--xp") p.xp = x;
            else if (a == "--yp") p.yp = x;
            else if (a == "--mesh-max-scale") p.mesh_max_scale = x;
            else if (a == "--steps") o.steps = (long long)x;
            else if (a == "--output-every") o.output_every = (int)x;
            else if (a == "--save-every") o.save_every = (int)x;
            else if (a == "--residual-every") o.residual_every = (int)x;
            else if (a == "--chunk") o.chunk = (int)x;
            else {
                fprintf(stderr, "lbm_main: unknown option %s\n", a.c_str());
                return false;
            }
        }
    }
    if (o.chunk < 2 || o.output_every < 0 || o.save_every < 0 || o.residual_every < 0) {
        fprintf(stderr, "lbm_main: --chunk >= 2 and non-negative intervals\n");
        return false;
    }
    return true;
}

int fail(lbm_t *h, const char *what, int rc)
{
    fprintf(stderr, "lbm_main: %s: status %d: %s\n", what, rc, lbm_last_error(h));
    if (h) lbm_destroy(h);
    return 1;
}

}  // namespace

int main(int argc, char **argv)
{
    lbm_params p;
    lbm_default_params(&p);
    Options o;
    if (!parse(argc, argv, p, o)) {
        usage(stderr);
        return 2;
    }
    lbm_t *h = nullptr;
    int rc = lbm_create(&p, &h);                                   // ini_mesh (main.f90:250)
    if (rc) return fail(nullptr, "lbm_create", rc);
    if ((rc = lbm_load_motion_table(h, o.motion.c_str())))         // main.f90:254-255
        return fail(h, "motion table", rc);
    if ((rc = lbm_init(h, nullptr, nullptr))) return fail(h, "init", rc);   // main.f90:292
    if ((rc = lbm_read_boundary(h, o.boundary_dir.c_str())))      // main.f90:293
        return fail(h, "read_boundary", rc);
    const std::string out = o.out + "/";
    std::vector<double> body(11 * (size_t)p.wing_count, 0.0);     // prescribed motion: no body state
    long long cycles = 0;   // force.dat rows of the run being continued (main.f90:263-274)
    if (!o.restart.empty()) {
        int cyc = 0, movenum = 0;
        const std::string dir = o.restart + "/";
        if ((rc = lbm_read_flow_field(h, (dir + "saved_flow_feild.dat").c_str(), &cyc, body.data(), &movenum)))
            return fail(h, "readflowfield", rc);
        cycles = count_lines(dir + "force.dat");
        const std::string f = out + "F" + std::to_string(cyc) + ".dat";   // output(n, mesh) after the restore
        if ((rc = lbm_write_tecplot(h, f.c_str(), cyc, 2, 2))) return fail(h, "output", rc);
        printf("restarted from step %d (%lld force rows before it)\n", cyc, cycles);
    }
    FILE *ff = fopen((out + "force.dat").c_str(), "w");
    FILE *fm = fopen((out + "airfoil_motion.dat").c_str(), "w");
    if (!ff || !fm) {
        fprintf(stderr, "lbm_main: cannot open force.dat / airfoil_motion.dat in %s\n", o.out.c_str());
        return fail(h, "outputs", LBM_ERR_IO);
    }
    const int row_len = lbm_force_row_length(h);
    std::vector<double> rows((size_t)o.chunk * row_len), mrow(1 + 3 * (size_t)p.wing_count, 0.0);
    const auto t0 = std::chrono::steady_clock::now();
    long long n = lbm_step_index(h), ran = 0;   // the next step's number (main.f90's n)
    const long long last = o.steps >= 0 ? o.steps : (long long)1 << 62;
    // the next step >= from at which the loop must stop for host work: the
    // output and checkpoint steps, and step k*R - 1, whose residual (of steps
    // k*R - 1 and k*R - 2) the reference computes at the start of step k*R
    auto next_event = [&](long long from) {
        long long e = last;
        auto upto = [&](long long every, long long off) {
            if (every <= 0) return;
            long long k = (from + off + every - 1) / every * every - off;
            if (k < from) k += every;
            e = std::min(e, k);
        };
        upto(o.output_every, 0);
        upto(o.save_every, 0);
        upto(o.residual_every, 1);
        return e;
    };
    while (n <= last) {
        const long long stop = std::min(next_event(n), n + o.chunk - 1);
        const int want = (int)(stop - n + 1);
        int done = 0;
        rc = lbm_run(h, want, rows.data(), &done);
        for (int k = 0; k < done; ++k) {
            const long long step = n + k;
            if (step <= cycles) continue;                            // rows already in the old force.dat
            const double *r = rows.data() + (size_t)k * row_len;
            fputs(f15_row(r, row_len).c_str(), ff);
            mrow[0] = r[0];                                         // time; body_extra_v/UU, body_extra_s*scale = 0
            fputs(f15_row(mrow.data(), (int)mrow.size()).c_str(), fm);
        }
        ran += done;
        n += done;
        if (rc == LBM_DONE) break;                                   // time > motion_end_time (main.f90:353)
        if (rc) {
            fclose(ff);
            fclose(fm);
            return fail(h, "evolution", rc);
        }
        const long long m = n - 1;                                   // the step just completed
        if (o.residual_every > 0 && (m + 1) % o.residual_every == 0 && m >= 1) {
            // erranalysis at the start of step m + 1, printed with that step's
            // number (main.f90:356-357, 391-393)
            double err = 0.0;
            if ((rc = lbm_residual(h, &err))) return fail(h, "erranalysis", rc);
            printf("iteration %lld, residual %.10e\n", m + 1, err);
        }
        if (o.output_every > 0 && m % o.output_every == 0 && (o.win_a < 0 || (m > o.win_a && m <= o.win_b))) {
            const std::string f = out + "F" + std::to_string(m) + ".dat";
            if ((rc = lbm_write_tecplot(h, f.c_str(), (int)m, 2, 2))) return fail(h, "output", rc);
        }
        if (o.save_every > 0 && m % o.save_every == 0) {          // saveflowfield (main.f90:413-416)
            fflush(ff);
            if ((rc = lbm_save_flow_field(h, (out + "saved_flow_feild.dat").c_str(), body.data(), 0)))
                return fail(h, "saveflowfield", rc);
        }
    }
    fclose(ff);
    fclose(fm);
    const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    printf("Run time = %.3f s, %lld steps, %.1f MLUPS\n", el, ran,
           ran > 0 ? (double)p.nx * p.ny * (double)ran / el / 1e6 : 0.0);
    lbm_destroy(h);
    return 0;
}
