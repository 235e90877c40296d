// Drop-in use of libcompact_b200 through the reference-shaped C++ API:
// numerics_pc<double>::deriv1d on a linear field (known answer of
// tests/test_numerics_serial.cu:60-131), physics::calc_fluxes /
// calc_viscous_shear_stress / calc_time_step on a Taylor-Green state with
// metric arrays, and one RK update.  Prints PASS/FAIL.
#include <cmath>
#include <cstdio>
#include <vector>

#include "compact_schemes.hpp"

int main() {
    const int nx = 64, ny = 32, nz = 16;
    t_dcomp d{nx * ny * nz, nx, ny, nz};
    const size_t n = (size_t)d.lmx;
    int nbc[2][3] = {{BC_NON_REFLECTIVE, BC_NON_REFLECTIVE, BC_NON_REFLECTIVE},
                     {BC_NON_REFLECTIVE, BC_NON_REFLECTIVE, BC_NON_REFLECTIVE}};
    numerics_pc<double> num(d, nbc);
    num.deriv_setup();
    std::vector<double> h(n);
    for (size_t i = 0; i < n; ++i) h[i] = (double)i;
    double *in, *out;
    cudaMalloc(&in, n * sizeof(double));
    cudaMalloc(&out, n * sizeof(double));
    cudaMemcpy(in, h.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    num.deriv1d<1>(in, out, 0, 0, d, 0);
    cudaMemcpy(h.data(), out, n * sizeof(double), cudaMemcpyDeviceToHost);
    double err = 0;
    for (size_t i = 0; i < n; ++i) err = std::fmax(err, std::fabs(h[i] - nx) / nx);
    std::printf("deriv1d<1> linear field rel err %.3e\n", err);
    bool ok = err < 1e-13;

    // periodic Taylor-Green state with uniform metrics as arrays
    int pbc[2][3] = {{BC_PERIODIC, BC_PERIODIC, BC_PERIODIC}, {BC_PERIODIC, BC_PERIODIC, BC_PERIODIC}};
    numerics_pc<double> pnum(d, pbc);
    pnum.deriv_setup();
    double *q, *de, *p, *xim, *etm, *zem, *yaco, *ssk, *q1;
    for (double **a : {&q, &de, &q1}) cudaMalloc(a, 5 * n * sizeof(double));
    for (double **a : {&xim, &etm, &zem}) cudaMalloc(a, 3 * n * sizeof(double));
    for (double **a : {&p, &yaco, &ssk}) cudaMalloc(a, n * sizeof(double));
    cs_tgv_init(q, nx, ny, nz, 0.1, 1e-4, 0, nullptr);
    const double tp = 6.283185307179586;
    const double hx = tp / nx, hy = tp / ny, hz = tp / nz;
    std::vector<double> m(3 * n, 0.0), one(n);
    for (int a = 0; a < 3; ++a) {
        const double diag = a == 0 ? hy * hz : (a == 1 ? hx * hz : hx * hy);
        std::fill(m.begin(), m.end(), 0.0);
        std::fill(m.begin() + a * n, m.begin() + (a + 1) * n, diag);
        cudaMemcpy(a == 0 ? xim : (a == 1 ? etm : zem), m.data(), 3 * n * sizeof(double), cudaMemcpyHostToDevice);
    }
    std::fill(one.begin(), one.end(), 1.0 / (hx * hy * hz));
    cudaMemcpy(yaco, one.data(), n * sizeof(double), cudaMemcpyHostToDevice);
    std::fill(one.begin(), one.end(), 0.1 / 1600.0);
    cudaMemcpy(ssk, one.data(), n * sizeof(double), cudaMemcpyHostToDevice);

    physics<true, double> phys(d);
    compact_b200::thermo(q, de, p, n);
    double dte = 0;
    phys.calc_time_step(xim, etm, zem, de, yaco, ssk, 0.5, &dte, (unsigned)n);
    cudaStream_t streams[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int mcd[2][3] = {{0, 0, 0}, {0, 0, 0}};
    phys.calc_viscous_shear_stress(de, ssk, xim, etm, zem, yaco, d, mcd, &pnum, streams);
    compact_b200::thermo(q, de, p, n);  // restore de[0], de[4] for the fluxes
    phys.calc_fluxes(q, p, de, xim, etm, zem, d, mcd, &pnum, streams);
    compact_b200::rk_update(q, de, yaco, dte / 4.0, q1, n);
    // wall state at the x faces if they were walls: every point of the mask is
    // a fluid point (npex = 1), so the state must not change
    {
        gcbc<double, int> gc(d);
        std::vector<int> fluid(n, 1);
        cudaMemcpy(gc.npex, fluid.data(), n * sizeof(int), cudaMemcpyHostToDevice);
        int wall[2][3] = {{BC_WALL_VISCOUS, BC_NON_REFLECTIVE, BC_NON_REFLECTIVE},
                          {BC_WALL_INVISCID, BC_NON_REFLECTIVE, BC_NON_REFLECTIVE}};
        t_point<double> umf0{0.0, 0.0, 0.0};
        wall_condition_update(q1, gc.npex, umf0, d, wall);
        cudaDeviceSynchronize();
    }
    std::vector<double> r(5 * n);
    cudaMemcpy(r.data(), q1, 5 * n * sizeof(double), cudaMemcpyDeviceToHost);
    double mass = 0;
    for (size_t i = 0; i < n; ++i) mass += r[i];
    const bool finite = std::isfinite(mass) && dte > 0 && dte < 1;
    std::printf("dt %.6e mass after one stage %.12f\n", dte, mass / n);
    ok = ok && finite && std::fabs(mass / n - 1.0) < 1e-3;
    std::printf("%s\n", ok ? "PASS" : "FAIL");
    return ok ? 0 : 1;
}
