// C++ consumer of include/neon_b200.hpp, the way a neon build would use it.  Prints one JSON
// object.
//   adapter_driver [n]   the linear-solver plugin on the 3x3 system of test/linear_solvers.cpp
//                        and a static_matrix solve of a linear elastic n^3 cube (bottom fixed,
//                        top uz = 1e-3)
//   adapter_driver --deck deck.json --mesh part.mesh [--step k] [--mixed]
//                  [--direct tolerance iterations] [--parse-only]
//                        one load step of a neon input deck through include/neon_b200_json.hpp
//                        (nlohmann::json, as neon uses): the part, its boundaries and loads, and
//                        static_matrix(mesh, simulation).solve(); --parse-only prints what the
//                        deck describes without touching the device.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/neon_b200.hpp"

#ifdef NB2_DRIVER_JSON
#include <fstream>
#include <string>

#include <nlohmann/json.hpp>

#include "../../include/neon_b200_json.hpp"

namespace {

using json = nlohmann::json;

json tables_json(std::vector<neon_b200::dof_table> const& tables) {
    json out = json::array();
    for (auto const& t : tables)
        out.push_back({{"dofs", t.dofs}, {"times", t.times}, {"values", t.values},
                       {"weights", t.weights}});
    return out;
}

int run_deck(int argc, char** argv) {
    std::string deck_path, mesh_path;
    int step = 0;
    bool parse_only = false;
    std::int32_t precision = NB2_FP64;
    neon_b200::direct_solver_substitute direct;
    for (int i = 1; i < argc; ++i) {
        std::string a = argv[i];
        if (a == "--deck" && i + 1 < argc) deck_path = argv[++i];
        else if (a == "--mesh" && i + 1 < argc) mesh_path = argv[++i];
        else if (a == "--step" && i + 1 < argc) step = std::atoi(argv[++i]);
        else if (a == "--mixed") precision = NB2_MIXED;
        else if (a == "--parse-only") parse_only = true;
        else if (a == "--direct" && i + 2 < argc) {
            direct.allowed = true;
            direct.tolerance = std::atof(argv[++i]);
            direct.maximum_iterations = std::atoi(argv[++i]);
        }
    }
    json deck, mesh_file;
    std::ifstream(deck_path) >> deck;
    std::ifstream(mesh_path) >> mesh_file;
    json out;
    try {
        json const& simulation = deck.at("steps").at(step);
        json const& mesh_data = simulation.at("meshes").front();
        json material;
        for (auto const& part : deck.at("parts"))
            if (part.at("name") == mesh_data.at("name"))
                for (auto const& m : deck.at("materials"))
                    if (m.at("name") == part.at("material")) material = m;
        neon_b200::basic_mesh part(mesh_file);
        double const dt = simulation.at("time").at("increments").at("initial").get<double>();
        if (parse_only) {
            auto const d = neon_b200::describe_mesh(part, material, mesh_data, dt);
            auto const o = neon_b200::make_solver_options(simulation, precision, direct);
            json loads = json::array();
            for (auto const& s : d.loads)
                loads.push_back({{"kind", s.kind}, {"component", s.component},
                                 {"faces", s.faces}, {"nodes_per_face", s.nodes_per_face},
                                 {"reduced", s.reduced_quadrature}, {"times", s.times},
                                 {"values", s.values}, {"name", s.name}});
            out = {{"nodes", part.nodes()},
                   {"connectivity", d.connectivity},
                   {"nodes_per_element", d.nodes_per_element},
                   {"material",
                    {d.material.model, d.material.bulk_modulus, d.material.shear_modulus,
                     d.material.yield_stress, d.material.isotropic_hardening_modulus,
                     d.material.segments_per_chain, d.material.nonaffine_stretch_parameter,
                     d.material.unit_sphere_points}},
                   {"options",
                    {o.residual_tolerance, o.displacement_tolerance, o.linear_iterations,
                     o.absolute_tolerance, o.period, o.initial_increment, o.minimum_increment,
                     o.maximum_increment, o.adaptive, o.cg_tolerance, o.cg_maximum_iterations}},
                   {"dirichlet", tables_json(d.dirichlet)},
                   {"nodal_forces", tables_json(d.nodal_forces)},
                   {"loads", loads}};
        } else {
            neon_b200::mesh m(part, material, mesh_data, dt);
            neon_b200::static_matrix solver(m, simulation, precision, direct);
            solver.solve();
            out = {{"u", solver.displacement()},
                   {"newton_iterations", solver.report().newton_iterations},
                   {"forces", tables_json(m.external_forces())}};
        }
    } catch (neon_b200::computational_error const& e) {
        out = {{"error", "computational_error"}, {"what", e.what()}};
    } catch (std::domain_error const& e) {
        out = {{"error", "domain_error"}, {"what", e.what()}};
    }
    std::printf("%s\n", out.dump().c_str());
    return 0;
}

}  // namespace
#endif

int main(int argc, char** argv) {
    if (argc > 1 && std::strcmp(argv[1], "--deck") == 0) {
#ifdef NB2_DRIVER_JSON
        return run_deck(argc, argv);
#else
        std::printf("{\"error\": \"built without nlohmann/json.hpp\"}\n");
        return 2;
#endif
    }
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
