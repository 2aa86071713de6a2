// imogen_run -- standalone driver of the library's fluid step: runs without Matlab and without
// Python, through the C ABI of include/imogen_b200.h only.
//
// It plays the part of the reference's own drivers: the Matlab main loop (imogen.m:115-139 with
// TimeManager.m:124-186, 270-277) and imogenCore's C++ loop (gpuimogen_core.cu:954-1054):
//   per iteration  tau = min over fluids of the CFL time (ib_cflTimestepFused)
//                  dt  = CFL * tau, clipped so that t + 2 dt <= t_max
//                  source(dt/2); fluid step forward; source(dt); fluid step backward; source(dt/2)
//                  t  += 2 dt (Kahan-compensated), iteration += 1
// where the source is the two-fluid drag (ib_cudaSource2FluidDrag) for the gas-dust problem and
// absent otherwise.
//
// Problems (initial states built here, or read from raw files with --input / --dust-input):
//   kh     Kelvin-Helmholtz shear layer in the periodic unit cube: rho = 2, v_x = +0.5 for
//          |y - 1/2| < 1/4, else rho = 1, v_x = -0.5; P = 2.5; gamma = 5/3; v perturbed by
//          U(-0.01, 0.01) per component from a counter-based hash of the cell index.
//   sod    Sod shock tube on [0, 1] along x: (rho, u, P) = (1, 0, 1) | (0.125, 0, 0.1) at x = 1/2,
//          gamma = 1.4, constant boundaries.
//   dusty  2-D periodic gas + dust: gas rho = 1, P = 1, v_y = 1e-3 sin(2 pi x) + U(+-1e-3),
//          v_x = U(+-1e-3), gamma = 5/3; dust at rest, rho_d / rho_g log-uniform in [0.01, 1],
//          isothermal c_s = 0.1 (gamma := 2), E = 1e-4 rho_d; drag between them.
// State files are the library's layout: 5 slabs [rho, E, px, py, pz] of slab_pitch doubles each
// (little-endian float64, x fastest).
//
// Output: one JSON line (problem, grid, iterations, simulated time, device milliseconds of the
// loop from CUDA events, Mcell-updates/s); --output / --dust-output write the final states.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "imogen_b200.h"

namespace {

struct Options {
    std::string problem = "kh";
    int grid[3] = {64, 64, 64};
    bool grid_set = false;
    int method = 2;  // 1 HLL, 2 HLLC, 3 Xin-Jin
    int slope = IB_SLOPE_MC;
    int fluxlim = IB_FLUX_OSPRE;
    int precision = IB_PREC_FP64;
    int drag = IB_DRAG_LOGTRAP2;
    double cfl = 0.4;
    long steps = 10;
    bool steps_set = false;
    double tmax = INFINITY;
    int device = 0;
    std::string input, dust_input, output, dust_output;
};

void usage(FILE *f)
{
    std::fprintf(f,
                 "usage: imogen_run [--problem kh|sod|dusty] [--grid nx,ny,nz] [--method hll|hllc|xj]\n"
                 "                  [--limiter mc|ospre|vanleer|minmod|superbee|vanalbada] [--precision fp64|fp32flux]\n"
                 "                  [--drag emp|rk4|etdrk1|etdrk2|logtrap2|logtrap3] [--cfl C] [--steps N] [--tmax T]\n"
                 "                  [--input gas.bin] [--dust-input dust.bin] [--output gas.bin] [--dust-output dust.bin]\n"
                 "                  [--device D]\n"
                 "Runs the library's fluid iterations (and the gas-dust drag for --problem dusty) and prints one JSON\n"
                 "line.  Defaults: kh on 64^3, HLLC, MC limiter, FP64, CFL 0.4, 10 iterations (sod: to t = 0.2).\n");
}

int lookup(const char *v, const char *const *names, const int *codes, int n)
{
    for (int i = 0; i < n; i++)
        if (!std::strcmp(v, names[i])) return codes[i];
    return -1;
}

// returns 0 on success, 1 for --help, 2 for a bad argument
int parse(int argc, char **argv, Options &o)
{
    for (int i = 1; i < argc; i++) {
        const char *a = argv[i];
        if (!std::strcmp(a, "--help") || !std::strcmp(a, "-h")) return 1;
        if (i + 1 >= argc) {
            std::fprintf(stderr, "imogen_run: %s needs a value\n", a);
            return 2;
        }
        const char *v = argv[++i];
        if (!std::strcmp(a, "--problem")) {
            o.problem = v;
            if (o.problem != "kh" && o.problem != "sod" && o.problem != "dusty") return 2;
        } else if (!std::strcmp(a, "--grid")) {
            if (std::sscanf(v, "%d,%d,%d", &o.grid[0], &o.grid[1], &o.grid[2]) != 3) return 2;
            if (o.grid[0] < 1 || o.grid[1] < 1 || o.grid[2] < 1) return 2;
            o.grid_set = true;
        } else if (!std::strcmp(a, "--method")) {
            static const char *const n[] = {"hll", "hllc", "xj"};
            static const int c[] = {1, 2, 3};
            if ((o.method = lookup(v, n, c, 3)) < 0) return 2;
        } else if (!std::strcmp(a, "--limiter")) {
            static const char *const n[] = {"mc", "ospre", "vanleer", "minmod", "superbee", "vanalbada"};
            static const int c[] = {IB_SLOPE_MC, IB_SLOPE_OSPRE, IB_SLOPE_VANLEER, IB_SLOPE_MINMOD, IB_SLOPE_SUPERBEE,
                                    IB_SLOPE_VANALBADA};
            if ((o.slope = lookup(v, n, c, 6)) < 0) return 2;
        } else if (!std::strcmp(a, "--precision")) {
            static const char *const n[] = {"fp64", "fp32flux"};
            static const int c[] = {IB_PREC_FP64, IB_PREC_FP32_FLUX};
            if ((o.precision = lookup(v, n, c, 2)) < 0) return 2;
        } else if (!std::strcmp(a, "--drag")) {
            static const char *const n[] = {"emp", "rk4", "etdrk1", "etdrk2", "logtrap2", "logtrap3"};
            static const int c[] = {IB_DRAG_EMP, IB_DRAG_RK4, IB_DRAG_ETDRK1, IB_DRAG_ETDRK2, IB_DRAG_LOGTRAP2,
                                    IB_DRAG_LOGTRAP3};
            if ((o.drag = lookup(v, n, c, 6)) < 0) return 2;
        } else if (!std::strcmp(a, "--cfl")) {
            o.cfl = std::atof(v);
            if (!(o.cfl > 0)) return 2;
        } else if (!std::strcmp(a, "--steps")) {
            o.steps = std::atol(v);
            if (o.steps < 0) return 2;
            o.steps_set = true;
        } else if (!std::strcmp(a, "--tmax")) {
            o.tmax = std::atof(v);
            if (!(o.tmax > 0)) return 2;
        } else if (!std::strcmp(a, "--device")) {
            o.device = std::atoi(v);
        } else if (!std::strcmp(a, "--input")) {
            o.input = v;
        } else if (!std::strcmp(a, "--dust-input")) {
            o.dust_input = v;
        } else if (!std::strcmp(a, "--output")) {
            o.output = v;
        } else if (!std::strcmp(a, "--dust-output")) {
            o.dust_output = v;
        } else {
            std::fprintf(stderr, "imogen_run: unknown option %s\n", a);
            return 2;
        }
    }
    if (!o.grid_set) {
        if (o.problem == "sod") { o.grid[0] = 1024; o.grid[1] = 1; o.grid[2] = 1; }
        if (o.problem == "dusty") { o.grid[0] = 512; o.grid[1] = 512; o.grid[2] = 1; }
    }
    if (o.problem == "sod" && !o.steps_set && !std::isfinite(o.tmax)) {
        o.tmax = 0.2;
        o.steps = -1;  // run to t_max
    }
    if (std::isfinite(o.tmax) && !o.steps_set) o.steps = -1;
    return 0;
}

// Uniform value in [-1, 1) from a 64-bit hash of (stream, index) (SplitMix64 finaliser).
double hash_uniform(uint64_t stream, uint64_t index)
{
    uint64_t z = index * 0x9E3779B97F4A7C15ull + stream * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

void fill_kh(const int g[3], int64_t S, std::vector<double> &q)
{
    const double gamma = 5.0 / 3.0, P0 = 2.5, amp = 1e-2;
    const int64_t nx = g[0], ny = g[1], nz = g[2];
    for (int64_t z = 0; z < nz; z++)
        for (int64_t y = 0; y < ny; y++)
            for (int64_t x = 0; x < nx; x++) {
                const int64_t i = (z * ny + y) * nx + x;
                const double yc = (y + 0.5) / ny;
                const bool band = std::fabs(yc - 0.5) < 0.25;
                const double rho = band ? 2.0 : 1.0;
                const double vx = (band ? 0.5 : -0.5) + amp * hash_uniform(1, i);
                const double vy = amp * hash_uniform(2, i);
                const double vz = nz > 1 ? amp * hash_uniform(3, i) : 0.0;
                q[i] = rho;
                q[S + i] = P0 / (gamma - 1) + 0.5 * rho * (vx * vx + vy * vy + vz * vz);
                q[2 * S + i] = rho * vx;
                q[3 * S + i] = rho * vy;
                q[4 * S + i] = rho * vz;
            }
}

void fill_sod(const int g[3], int64_t S, std::vector<double> &q)
{
    const double gamma = 1.4;
    const int64_t nx = g[0], n = (int64_t)g[0] * g[1] * g[2];
    for (int64_t i = 0; i < n; i++) {
        const double xc = ((i % nx) + 0.5) / nx;
        const bool left = xc < 0.5;
        const double rho = left ? 1.0 : 0.125, P = left ? 1.0 : 0.1;
        q[i] = rho;
        q[S + i] = P / (gamma - 1);
        q[2 * S + i] = q[3 * S + i] = q[4 * S + i] = 0.0;
    }
}

void fill_dusty(const int g[3], int64_t S, std::vector<double> &gas, std::vector<double> &dust)
{
    const double gamma = 5.0 / 3.0, pi = 3.141592653589793;
    const int64_t nx = g[0], n = (int64_t)g[0] * g[1] * g[2];
    for (int64_t i = 0; i < n; i++) {
        const double xc = ((i % nx) + 0.5) / nx;
        const double vx = 1e-3 * hash_uniform(11, i);
        const double vy = 1e-3 * std::sin(2 * pi * xc) + 1e-3 * hash_uniform(12, i);
        gas[i] = 1.0;
        gas[S + i] = 1.0 / (gamma - 1) + 0.5 * (vx * vx + vy * vy);
        gas[2 * S + i] = vx;
        gas[3 * S + i] = vy;
        gas[4 * S + i] = 0.0;
        const double rd = std::exp(std::log(0.01) * 0.5 * (1.0 - hash_uniform(13, i)));
        dust[i] = rd;
        dust[S + i] = 1e-4 * rd;
        dust[2 * S + i] = dust[3 * S + i] = dust[4 * S + i] = 0.0;
    }
}

bool read_state(const std::string &path, std::vector<double> &q)
{
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    const size_t got = std::fread(q.data(), sizeof(double), q.size(), f);
    const bool more = std::fgetc(f) != EOF;
    std::fclose(f);
    return got == q.size() && !more;
}

bool write_state(const std::string &path, const std::vector<double> &q)
{
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const size_t put = std::fwrite(q.data(), sizeof(double), q.size(), f);
    return std::fclose(f) == 0 && put == q.size();
}

// Time bookkeeping of TimeManager.m:124-186 (dt = CFL tau, last-step clip) and :270-277
// (iteration += 1, Kahan-compensated t += 2 dt).
struct TimeManager {
    double cfl, tmax, time = 0, dtime = 0, kahan = 0;
    long iteration = 0, itermax;
    double update(double tau)
    {
        dtime = cfl * tau;
        if (time + 2 * dtime > tmax) dtime = .5 * (tmax - time);
        return dtime;
    }
    void step()
    {
        iteration++;
        const double y = (2 * dtime) - kahan;
        const double t = time + y;
        kahan = (t - time) - y;
        time = t;
    }
    bool running() const
    {
        if (itermax >= 0 && iteration >= itermax) return false;
        return std::isfinite(tmax) ? time < tmax * (1 - 1e-14) : true;
    }
};

int fail(const char *what, int status)
{
    std::fprintf(stderr, "imogen_run: %s failed: %s (%d), CUDA error %d\n", what, ib_status_string(status), status,
                 ib_last_cuda_error());
    return 3;
}

}  // namespace

int main(int argc, char **argv)
{
    Options o;
    const int pr = parse(argc, argv, o);
    if (pr == 1) {
        usage(stdout);
        return 0;
    }
    if (pr) {
        usage(stderr);
        return 2;
    }
    const bool dusty = o.problem == "dusty";
    const int64_t S = ib_slab_pitch(o.grid[0], o.grid[1], o.grid[2]);
    const int64_t N = (int64_t)o.grid[0] * o.grid[1] * o.grid[2];
    std::vector<double> hq(5 * S, 0.0), hd(dusty ? 5 * S : 0, 0.0);
    if (!o.input.empty()) {
        if (!read_state(o.input, hq)) {
            std::fprintf(stderr, "imogen_run: %s is not a %lld-double state\n", o.input.c_str(), (long long)(5 * S));
            return 2;
        }
    } else if (o.problem == "kh") {
        fill_kh(o.grid, S, hq);
    } else if (o.problem == "sod") {
        fill_sod(o.grid, S, hq);
    }
    if (dusty) {
        std::vector<double> g0(5 * S, 0.0), d0(5 * S, 0.0);
        fill_dusty(o.grid, S, g0, d0);
        if (o.input.empty()) hq = g0;
        if (!o.dust_input.empty()) {
            if (!read_state(o.dust_input, hd)) {
                std::fprintf(stderr, "imogen_run: %s is not a state\n", o.dust_input.c_str());
                return 2;
            }
        } else {
            hd = d0;
        }
    }

    if (cudaSetDevice(o.device) != cudaSuccess) {
        std::fprintf(stderr, "imogen_run: no CUDA device %d\n", o.device);
        return 3;
    }
    const size_t bytes = sizeof(double) * 5 * S;
    double *dq = nullptr, *dd = nullptr;
    if (cudaMalloc(&dq, bytes) != cudaSuccess || (dusty && cudaMalloc(&dd, bytes) != cudaSuccess)) {
        std::fprintf(stderr, "imogen_run: cannot allocate %zu bytes per fluid\n", bytes);
        return 3;
    }
    cudaMemcpy(dq, hq.data(), bytes, cudaMemcpyHostToDevice);
    if (dusty) cudaMemcpy(dd, hd.data(), bytes, cudaMemcpyHostToDevice);

    // fluids, thermodynamics, geometry, numerics
    ib_fluid fl[2];
    std::memset(fl, 0, sizeof(fl));
    ib_fluid_thermo th[2];
    const int bcmode = (o.problem == "sod") ? IB_BC_CONST : IB_BC_CIRCULAR;
    for (int k = 0; k < 2; k++) {
        fl[k].grid.nx = o.grid[0];
        fl[k].grid.ny = o.grid[1];
        fl[k].grid.nz = o.grid[2];
        fl[k].grid.slab_pitch = S;
        for (int b = 0; b < 6; b++) fl[k].bc[b] = bcmode;
        fl[k].halo = 4;
    }
    fl[0].q = dq;
    fl[1].q = dd;
    const double gamma_gas = (o.problem == "sod") ? 1.4 : 5.0 / 3.0;
    th[0] = ib_fluid_thermo{gamma_gas, 1e-5, -1.0};
    th[1] = ib_fluid_thermo{2.0, 1e-5, 0.1};  // dust: isothermal, gamma := 2
    const int nfl = dusty ? 2 : 1;
    ib_geometry geo;
    std::memset(&geo, 0, sizeof(geo));
    for (int d = 0; d < 3; d++) {
        geo.h[d] = 1.0 / o.grid[d];
        geo.global_rez[d] = o.grid[d];
    }
    ib_numerics num{o.slope, o.fluxlim, o.precision, 0};
    // drag microphysics (gas: molecular hydrogen-like; dust: 0.1 um grains of mass 3e-19)
    const ib_thermo tgas{5.0 / 3.0, 3.3e-27, 8.4e-6, 0.7, 2.4e-19, 0.2, 1.381e-23, -1.0};
    const ib_thermo tdust{1.01, 3e-19, 0.0, 0.0, 3.141592653589793 * 25e-12, 0.0, 1.381e-23, 0.1};

    TimeManager tm{o.cfl, o.tmax};
    tm.itermax = o.steps;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto drag = [&](double dt) {
        const double p[2] = {dt, (double)o.drag};
        return ib_cudaSource2FluidDrag(&fl[0], &fl[1], &tgas, &tdust, &geo, p, 2, nullptr);
    };
    int rc = 0;
    cudaEventRecord(e0);
    while (tm.running()) {
        double tau = 1e38;
        for (int k = 0; k < nfl; k++) {
            double t = 0;
            rc = ib_cflTimestepFused(&fl[k], th[k].gamma, &geo, o.method, &t, nullptr, nullptr);
            if (rc) return fail("ib_cflTimestepFused", rc);
            if (!std::isfinite(t)) {
                std::fprintf(stderr, "imogen_run: non-finite timestep at iteration %ld\n", tm.iteration);
                return 4;
            }
            tau = std::fmin(tau, t);
        }
        const double dt = tm.update(tau);
        const double fwd[5] = {dt, 1, 1, (double)tm.iteration, (double)o.method};
        const double bwd[5] = {dt, 1, -1, (double)tm.iteration, (double)o.method};
        if (dusty && (rc = drag(0.5 * dt))) return fail("ib_cudaSource2FluidDrag", rc);
        if ((rc = ib_fluidstep(fl, th, nfl, &geo, fwd, 5, &num, nullptr))) return fail("ib_fluidstep", rc);
        if (dusty && (rc = drag(dt))) return fail("ib_cudaSource2FluidDrag", rc);
        if ((rc = ib_fluidstep(fl, th, nfl, &geo, bwd, 5, &num, nullptr))) return fail("ib_fluidstep", rc);
        if (dusty && (rc = drag(0.5 * dt))) return fail("ib_cudaSource2FluidDrag", rc);
        tm.step();
    }
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) return fail("the iteration loop", IB_ERROR_CUDA);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    const int wait = ib_device_wait_status(0);
    if (wait != 0) {
        std::fprintf(stderr, "imogen_run: a sweep's tile wait ran out (%d)\n", wait);
        return 3;
    }

    cudaMemcpy(hq.data(), dq, bytes, cudaMemcpyDeviceToHost);
    if (dusty) cudaMemcpy(hd.data(), dd, bytes, cudaMemcpyDeviceToHost);
    if (!o.output.empty() && !write_state(o.output, hq)) {
        std::fprintf(stderr, "imogen_run: cannot write %s\n", o.output.c_str());
        return 2;
    }
    if (dusty && !o.dust_output.empty() && !write_state(o.dust_output, hd)) {
        std::fprintf(stderr, "imogen_run: cannot write %s\n", o.dust_output.c_str());
        return 2;
    }
    double mass = 0;
    for (int64_t i = 0; i < N; i++) mass += hq[i];
    const double rate = (ms > 0) ? (double)N * tm.iteration / (ms * 1e-3) / 1e6 : 0.0;
    std::printf("{\"problem\": \"%s\", \"grid\": [%d, %d, %d], \"iterations\": %ld, \"time\": %.17g, "
                "\"ms\": %.4f, \"mcell_updates_per_s\": %.2f, \"gas_mass\": %.17g, \"launches\": %lld}\n",
                o.problem.c_str(), o.grid[0], o.grid[1], o.grid[2], tm.iteration, tm.time, ms, rate, mass,
                ib_launch_count());
    cudaFree(dq);
    if (dd) cudaFree(dd);
    return 0;
}
