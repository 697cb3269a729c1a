// Uses the C++ reverse-mode API (include/fvgpu_adjoint.hpp) on a mesh file:
//   adjoint_api <mesh.msh> <steps> <theta_0> ... <theta_nb>
// prints "loss g_0 ... g_nb" with 17 significant digits, or "error: <message>"
// (exit code 3) when the library refuses (e.g. no CUDA device).
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "fvgpu_adjoint.hpp"

int main(int argc, char** argv) {
    if (argc < 4) return 2;
    fv_mesh* m = nullptr;
    if (fv_mesh_read_msh(argv[1], &m) != FV_OK) {
        std::printf("error: %s\n", fv_last_error());
        return 3;
    }
    // groups in the file: wall, inlet, outlet, step (forward-step mesh)
    const int32_t bc[4] = {FV_BC_WALL, FV_BC_INLET_OUTLET, FV_BC_INLET_OUTLET, FV_BC_WALL};
    // inflow state of examples/forwardStep/main.cpp:196-201 (same arithmetic)
    const double gamma = 1.4, bv0 = 1.4, bv1 = bv0 * 3.0, bv2 = bv0 * 0.0;
    const double bv3 = 1.0 / (gamma - 1) + 0.5 / bv0 * (bv1 * bv1 + bv2 * bv2);
    const double bv[16] = {0, 0, 0, 0, bv0, bv1, bv2, bv3, bv0, bv1, bv2, bv3, 0, 0, 0, 0};
    fv_physics ph = {4, FV_FLUX_ROE_FS, 1, FV_LIM_VENKAT, FV_DT_CFL_SUM, 1, 1.4, 5.0, 0.8, 0.0, 4, bc, bv, 1};
    const double alpha[5] = {0.0695, 0.1602, 0.2898, 0.506, 1.0};
    std::vector<double> theta;
    for (int i = 3; i < argc; ++i) theta.push_back(std::atof(argv[i]));
    fv_adjoint_options o = {std::atoi(argv[2]), 10, 5, alpha, 3, 1, (int32_t)theta.size() - 1, 0.0, 1.0};
    try {
        fvgpu::InflowAdjoint adj(m, ph, o, 0);
        double loss = 0.0;
        std::vector<double> g = adj.gradient(theta, &loss);
        std::printf("%.17g", loss);
        for (double v : g) std::printf(" %.17g", v);
        std::printf("\n");
    } catch (const std::exception& ex) {
        std::printf("error: %s\n", ex.what());
        fv_mesh_destroy(m);
        return 3;
    }
    fv_mesh_destroy(m);
    return 0;
}
