// The reference driver's time loop (driver/canard.cu:97-224) written against
// the drop-in headers, call for call: physics<true, Type>, numerics_pc<Type>,
// deriv_setup, movef, calc_time_step, calc_viscous_shear_stress, calc_fluxes,
// gcbc<Type, int> + gcbc_go(numerics_instance.drva_buffer, d_cm,
// gcbc_instance.drvb, ...) and wall_condition_update, with the conserved
// update that movef leaves empty.  Type is double: the drop-in physics path
// is FP64 (the reference instantiates float).  The grid and domain
// decomposition objects are stand-ins holding what the loop reads (metric
// arrays, nbc, mcd).  Box: 48 x 32 x 16 Taylor-Green state, non-reflective x
// faces, viscous walls on y, periodic z.  Prints PASS when the state stays
// finite and the walls hold their no-slip momentum.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "compact_schemes.hpp"

using Type = double;

struct grid_standin {
    Type *xim, *etm, *zem;
};
struct domdcomp_standin {
    int nbc[2][3];
    int mcd[2][3];
};

int main() {
    const int nx = 48, ny = 32, nz = 16;
    t_dcomp dcomp_info{nx * ny * nz, nx, ny, nz};
    const size_t n = (size_t)dcomp_info.lmx;
    domdcomp_standin domdcomp_instance{{{BC_NON_REFLECTIVE, BC_WALL_VISCOUS, BC_PERIODIC},
                                        {BC_NON_REFLECTIVE, BC_WALL_VISCOUS, BC_PERIODIC}},
                                       {{0, 0, 0}, {0, 0, 0}}};
    int mcd[2][3] = {{0, 0, 0}, {0, 0, 0}};

    Type *d_qa, *d_de, *d_pressure, *d_yaco, *d_ss, *d_qn;
    int *d_npex;
    cudaMalloc(&d_qa, 5 * n * sizeof(Type));
    cudaMalloc(&d_qn, 5 * n * sizeof(Type));
    cudaMalloc(&d_de, 5 * n * sizeof(Type));
    cudaMalloc(&d_pressure, n * sizeof(Type));
    cudaMalloc(&d_yaco, n * sizeof(Type));
    cudaMalloc(&d_ss, n * sizeof(Type));
    cudaMalloc(&d_npex, n * sizeof(int));

    // uniform grid of spacing h: xim = (h^2, 0, 0) etc., yaco = 1 / h^3
    const Type h = 6.283185307179586 / nx;
    grid_standin grid_instance;
    cudaMalloc(&grid_instance.xim, 3 * n * sizeof(Type));
    cudaMalloc(&grid_instance.etm, 3 * n * sizeof(Type));
    cudaMalloc(&grid_instance.zem, 3 * n * sizeof(Type));
    std::vector<Type> m(3 * n);
    for (int a = 0; a < 3; ++a) {
        std::fill(m.begin(), m.end(), 0.0);
        std::fill(m.begin() + a * n, m.begin() + (a + 1) * n, h * h);
        cudaMemcpy(a == 0 ? grid_instance.xim : (a == 1 ? grid_instance.etm : grid_instance.zem), m.data(),
                   3 * n * sizeof(Type), cudaMemcpyHostToDevice);
    }
    std::vector<Type> one(n, 1.0 / (h * h * h));
    cudaMemcpy(d_yaco, one.data(), n * sizeof(Type), cudaMemcpyHostToDevice);
    std::fill(one.begin(), one.end(), 0.1 / 1600.0);
    cudaMemcpy(d_ss, one.data(), n * sizeof(Type), cudaMemcpyHostToDevice);
    // wall mask: 0 on the y faces (wall points), 1 elsewhere
    std::vector<int> npex(n, 1);
    for (int k = 0; k < nz; ++k)
        for (int i = 0; i < nx; ++i) {
            npex[i + (size_t)nx * (0 + (size_t)ny * k)] = 0;
            npex[i + (size_t)nx * ((ny - 1) + (size_t)ny * k)] = 0;
        }
    cudaMemcpy(d_npex, npex.data(), n * sizeof(int), cudaMemcpyHostToDevice);
    cs_tgv_init(d_qa, nx, ny, nz, 0.1, 1e-4, 0, nullptr);

    // face normals of the GCBC faces and the boundary weights sbcc = 1/J on
    // the face planes
    Type *d_cm[3];
    const size_t F[3] = {(size_t)ny * nz, (size_t)nx * nz, (size_t)nx * ny};
    for (int a = 0; a < 3; ++a) {
        cudaMalloc(&d_cm[a], 6 * F[a] * sizeof(Type));
        std::vector<Type> c(6 * F[a], 0.0);
        for (int ip = 0; ip < 2; ++ip) std::fill(c.begin() + (ip * 3 + a) * F[a], c.begin() + (ip * 3 + a + 1) * F[a], 1.0);
        cudaMemcpy(d_cm[a], c.data(), c.size() * sizeof(Type), cudaMemcpyHostToDevice);
    }

    auto physics_instance = physics<true, Type>(dcomp_info);
    auto numerics_instance = numerics_pc<Type>(dcomp_info, domdcomp_instance.nbc);
    numerics_instance.deriv_setup();
    auto gcbc_instance = gcbc<Type, int>(dcomp_info);
    {
        std::vector<Type> s(n, 0.0);
        for (size_t i = 0; i < n; ++i) {
            const size_t ii = i % nx, jj = (i / nx) % ny;
            if (ii == 0 || ii == (size_t)nx - 1 || jj == 0 || jj == (size_t)ny - 1) s[i] = h * h * h;
        }
        cudaMemcpy(gcbc_instance.sbcc, s.data(), n * sizeof(Type), cudaMemcpyHostToDevice);
    }

    cudaStream_t stream[5];
    for (int i = 0; i < 5; i++) cudaStreamCreate(&stream[i]);

    Type dt = 0.0, dte = 0.0, timo = 0.0, cfl = 0.5, dtk, dtko;
    t_point<Type> umf{0, 0, 0}, dudtmf{0, 0, 0};
    physics_instance.init();
    for (int step = 0; step < 3; ++step) {
        cudaMemcpy(d_qn, d_qa, 5 * n * sizeof(Type), cudaMemcpyDeviceToDevice);
        for (int nk = 0; nk < nkrk; ++nk) {
            dtko = dt * std::min(std::max(nk - 2, 0), 1) / (nkrk - nk + 3);
            dtk = dt * std::min(nk - 1, 1) / (nkrk - nk + 2);
            physics_instance.movef(dtko, dtk, timo);

            compact_b200::thermo(d_qa, d_de, d_pressure, n);
            if (nk == 0) {
                physics_instance.calc_time_step(grid_instance.xim, grid_instance.etm, grid_instance.zem, d_de,
                                                d_yaco, d_ss, cfl, &dte, dcomp_info.lmx);
                dt = dte;
            }

            physics_instance.calc_viscous_shear_stress(d_de, d_ss, grid_instance.xim, grid_instance.etm,
                                                       grid_instance.zem, d_yaco, dcomp_info,
                                                       domdcomp_instance.mcd, &numerics_instance, &stream[0]);
            compact_b200::thermo(d_qa, d_de, d_pressure, n);
            physics_instance.calc_fluxes(d_qa, d_pressure, d_de, grid_instance.xim, grid_instance.etm,
                                         grid_instance.zem, dcomp_info, domdcomp_instance.mcd, &numerics_instance,
                                         &stream[0]);

            Type dtwi = 1 / dt;
            gcbc_go(numerics_instance.drva_buffer, d_cm, gcbc_instance.drvb, d_qa, d_de, d_pressure, d_yaco,
                    gcbc_instance.sbcc, umf, dudtmf, dcomp_info, dtwi, domdcomp_instance.nbc, mcd);

            // the stage coefficient dt / (4 - k): the driver's dt / (nkrk - nk + 1)
            // with its 0-based nk gives 1/5 .. 1/2 (driver/canard.cu:199)
            dtko = dt * std::min(nk - 1, 1) / (nkrk - nk + 2);
            dtk = dt / (nkrk - nk);
            physics_instance.movef(dtko, dtk, timo);
            compact_b200::rk_update(d_qn, d_de, d_yaco, dtk, d_qa, n);

            wall_condition_update(d_qa, d_npex, umf, dcomp_info, domdcomp_instance.nbc);
        }
        timo += dt;
    }
    cudaDeviceSynchronize();

    std::vector<Type> q(5 * n);
    cudaMemcpy(q.data(), d_qa, 5 * n * sizeof(Type), cudaMemcpyDeviceToHost);
    bool finite = true;
    for (Type v : q) finite = finite && std::isfinite(v);
    Type wall_mom = 0.0;
    for (size_t i = 0; i < n; ++i)
        if (npex[i] == 0)
            for (int v = 1; v <= 3; ++v) wall_mom = std::fmax(wall_mom, std::fabs(q[v * n + i]));
    const bool ok = finite && wall_mom == 0.0 && dt > 0.0 && cudaGetLastError() == cudaSuccess;
    std::printf("driver sequence: dt %.6e, finite %d, wall momentum %.3e\n", dt, (int)finite, wall_mom);
    std::printf("%s\n", ok ? "PASS" : "FAIL");

    for (int i = 0; i < 5; i++) cudaStreamDestroy(stream[i]);
    for (Type *a : {d_qa, d_qn, d_de, d_pressure, d_yaco, d_ss, grid_instance.xim, grid_instance.etm,
                    grid_instance.zem, d_cm[0], d_cm[1], d_cm[2]})
        cudaFree(a);
    cudaFree(d_npex);
    return ok ? 0 : 1;
}
