// C++ consumer of include/neon_b200.hpp, the way a neon build would use it: the linear-solver
// plugin on the 3x3 system of test/linear_solvers.cpp and a static_matrix solve of a linear
// elastic n^3 cube (bottom fixed, top uz = 1e-3).  Prints one JSON object.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../../include/neon_b200.hpp"

int main(int argc, char** argv) {
    int n = argc > 1 ? std::atoi(argv[1]) : 4;
    // --- linear solver plugin ---
    std::vector<std::int32_t> rp{0, 3, 6, 9}, col{0, 1, 2, 0, 1, 2, 0, 1, 2};
    std::vector<double> val{2, -1, 0, -1, 2, -1, 0, -1, 2}, b{1.0, 0.5, 1.5}, x;
    neon_b200::conjugate_gradient cg(1e-10, 100);
    cg.solve(3, rp.data(), col.data(), val.data(), x, b);
    bool threw = false;
    try {
        neon_b200::conjugate_gradient(1e-14, 1).solve(3, rp.data(), col.data(), val.data(), x, b);
    } catch (neon_b200::computational_error const&) {
        threw = true;
    }
    cg.solve(3, rp.data(), col.data(), val.data(), x, b);
    // --- static_matrix on a structured cube ---
    const int N1 = n + 1;
    std::vector<double> X;
    for (int k = 0; k <= n; ++k)
        for (int j = 0; j <= n; ++j)
            for (int i = 0; i <= n; ++i) {
                X.push_back(double(i) / n);
                X.push_back(double(j) / n);
                X.push_back(double(k) / n);
            }
    auto id = [&](int i, int j, int k) { return i + N1 * (j + N1 * k); };
    std::vector<std::int32_t> conn;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                for (int c : {id(i, j, k), id(i + 1, j, k), id(i + 1, j + 1, k), id(i, j + 1, k),
                              id(i, j, k + 1), id(i + 1, j, k + 1), id(i + 1, j + 1, k + 1),
                              id(i, j + 1, k + 1)})
                    conn.push_back(c);
    const double E = 200e3, nu = 0.3;
    nb2_material mat{NB2_ISOTROPIC_LINEAR_ELASTICITY, E / (3 * (1 - 2 * nu)), E / (2 * (1 + nu)),
                     0, 0, 0};
    neon_b200::solid_mesh mesh(X, conn, 8, mat);
    neon_b200::dof_table bx, by, bz, top;
    for (int j = 0; j <= n; ++j)
        for (int i = 0; i <= n; ++i) {
            bx.dofs.push_back(3 * id(i, j, 0) + 0);
            by.dofs.push_back(3 * id(i, j, 0) + 1);
            bz.dofs.push_back(3 * id(i, j, 0) + 2);
            top.dofs.push_back(3 * id(i, j, n) + 2);
        }
    for (auto* t : {&bx, &by, &bz}) {
        t->times = {0.0, 1.0};
        t->values = {0.0, 0.0};
    }
    top.times = {0.0, 1.0};
    top.values = {0.0, 1e-3};
    nb2_solver_options o{};
    o.residual_tolerance = o.displacement_tolerance = 1e-6;
    o.linear_iterations = 10;
    o.period = o.initial_increment = o.minimum_increment = o.maximum_increment = 1.0;
    o.cg_tolerance = 1e-10;
    o.cg_maximum_iterations = 100000;
    o.precision = NB2_FP64;
    o.use_graphs = 1;
    neon_b200::static_matrix sm(mesh, o, {bx, by, bz, top});
    sm.solve();
    auto const& u = sm.displacement();
    std::printf("{\"cg_x\": [%.17g, %.17g, %.17g], \"cg_iterations\": %d, \"maxit_threw\": %s, "
                "\"newton_iterations\": %lld, \"u\": [",
                x[0], x[1], x[2], cg.iterations(), threw ? "true" : "false",
                (long long)sm.report().newton_iterations);
    for (size_t i = 0; i < u.size(); ++i) std::printf("%s%.17g", i ? ", " : "", u[i]);
    std::printf("]}\n");
    return 0;
}
