// Compiles the C++ drop-in header the way a reference caller would use it and,
// when run on a GPU, solves the heat 64-row sweep through TdmaBackendGPU,
// PaScaLTDMACUDA and FilteredTDMACUDA (and, read as 512 x 512, both tiled
// kernel shapes), then the fused heat step and a ragged batch through the RAII
// wrappers.  Prints one line per solve:
//   <name> <max |x|> <status>
// tests/test_cpp_dropin.py compares the solutions with the oracle.
#include <cuda_runtime_api.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "btdma.hpp"

static void fill(std::vector<double>& A, std::vector<double>& B, std::vector<double>& C,
                 std::vector<double>& D, int n_sys, int n_row) {
    unsigned long long s = 12345;
    for (int j = 0; j < n_row; ++j)
        for (int i = 0; i < n_sys; ++i) {
            size_t k = (size_t)j * n_sys + i;
            A[k] = -1.0;
            C[k] = -1.0;
            B[k] = 3.0;
            s = s * 6364136223846793005ULL + 1442695040888963407ULL;
            D[k] = (double)(s >> 11) / 9007199254740992.0 * 2.0 - 1.0;
        }
}

int main(int argc, char** argv) {
    const int n_sys = 4096, n_row = 64;
    const size_t n = (size_t)n_sys * n_row;
    std::vector<double> A(n), B(n), C(n), D(n), X(n);
    fill(A, B, C, D, n_sys, n_row);
    if (argc > 1) {  // dump the inputs for the checker
        FILE* f = std::fopen(argv[1], "wb");
        std::fwrite(D.data(), sizeof(double), n, f);
        std::fclose(f);
    }
    double *dA, *dB, *dC, *dD;
    cudaMalloc((void**)&dA, n * 8);
    cudaMalloc((void**)&dB, n * 8);
    cudaMalloc((void**)&dC, n * 8);
    cudaMalloc((void**)&dD, n * 8);
    auto upload = [&] {
        cudaMemcpy(dA, A.data(), n * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, B.data(), n * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(dC, C.data(), n * 8, cudaMemcpyHostToDevice);
        cudaMemcpy(dD, D.data(), n * 8, cudaMemcpyHostToDevice);
    };
    auto report = [&](const char* name) {
        cudaMemcpy(X.data(), dD, n * 8, cudaMemcpyDeviceToHost);
        if (argc > 2) {
            char path[512];
            std::snprintf(path, sizeof path, "%s_%s.bin", argv[2], name);
            FILE* f = std::fopen(path, "wb");
            std::fwrite(X.data(), sizeof(double), n, f);
            std::fclose(f);
        }
        double m = 0;
        for (double v : X) m = std::fmax(m, std::fabs(v));
        std::printf("%s %.17g\n", name, m);
    };
    try {
        const char* kinds[] = {"pascal", "filtered", "filtered_v2"};
        for (const char* k : kinds) {
            upload();
            TdmaBackendGPU be(TdmaBackendGPU::parse(k), n_sys, n_row, 0, 4, 0, -2, -2, 1.0e-3);
            be.set_rho_device(dA, dB, dC);
            be.solve(dA, dB, dC, dD);
            report(k);
        }
        upload();
        PaScaLTDMACUDA p(n_sys, 0, 1);
        p.solve(dA, dB, dC, dD, n_sys, n_row);
        report("pascal_p1");
        upload();
        FilteredTDMACUDA f(n_sys, n_row, 0, 4, 0, -2, -2, 1.0e-3);
        f.set_rho_device(dA, dB, dC);
        f.solve_cycl_filtered_v2(dA, dB, dC, dD);
        report("filtered_v2_cyclic");
        std::printf("J %d\n", f.last_J());
        // the reference's interface also where J >= m - 2 (no exact fallback)
        upload();
        FilteredTDMACUDA fr(n_sys, n_row, 0, 4, 0, -2, -2, 1.0e-3, BTDMA_FLAG_REFERENCE_ORDER);
        fr.set_rho_device(dA, dB, dC);
        fr.solve_filtered_v2(dA, dB, dC, dD);
        report("filtered_v2_reference");
        // the same values read as 512 systems of 512 rows, through both tiled
        // kernel shapes
        for (int shape : {BTDMA_TILE_NARROW, BTDMA_TILE_WIDE}) {
            upload();
            PaScaLTDMACUDA w(512, 0, 8);
            w.set_tile_shape(shape);
            w.solve(dA, dB, dC, dD, 512, 512);
            report(shape == BTDMA_TILE_WIDE ? "pascal512_wide" : "pascal512_narrow");
        }

        // the fused heat step of the reference's order-accuracy run (32^3,
        // rho = 0.25, one step) through the C++ wrapper
        {
            const int g = 32;
            const double dx = 2.0 / g, rho = 0.25;
            const double dt = rho / (1.0 - 2.0 * rho) * (2.0 * dx * dx);
            double* th;
            cudaMalloc((void**)&th, sizeof(double) * (g + 2) * (g + 2) * (g + 2));
            btdma::HeatADI heat(g, g, g, dt);
            heat.init(th);
            heat.step(th, 1);
            std::printf("heat_l2 %.9g\n", heat.l2_error(th, dt));
            cudaFree(th);
        }
        // a small ragged batch: two systems of 5 and 40 rows, the second periodic
        {
            const long long off[3] = {0, 5, 45};
            const unsigned char per[2] = {0, 1};
            std::vector<double> ra(45, -1.0), rb(45, 4.0), rc(45, -1.0), rd(45, 1.0), rx(45);
            double *qa, *qb, *qc, *qd, *qx;
            for (double** p : {&qa, &qb, &qc, &qd, &qx}) cudaMalloc((void**)p, 45 * 8);
            cudaMemcpy(qa, ra.data(), 45 * 8, cudaMemcpyHostToDevice);
            cudaMemcpy(qb, rb.data(), 45 * 8, cudaMemcpyHostToDevice);
            cudaMemcpy(qc, rc.data(), 45 * 8, cudaMemcpyHostToDevice);
            cudaMemcpy(qd, rd.data(), 45 * 8, cudaMemcpyHostToDevice);
            btdma::RaggedSolver rs(2);
            rs.solve(qa, qb, qc, qd, qx, off, per, 2);
            rs.set_plan(rs.plan());  // a stored plan applied again
            rs.solve(qa, qb, qc, qd, qx, off, per, 2);
            cudaMemcpy(rx.data(), qx, 45 * 8, cudaMemcpyDeviceToHost);
            // periodic system of constant rows: x = 1 / (4 - 2) everywhere
            std::printf("ragged_periodic_x %.17g\n", rx[20]);
            for (double* p : {qa, qb, qc, qd, qx}) cudaFree(p);
        }
    } catch (const btdma::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
    return 0;
}
