// neon_b200.hpp -- C++ host adapter over the C-ABI (include/neon_b200.h).
//
// Header-only; the classes keep the names, argument meaning and error behaviour of neon's
// interfaces on this path so a neon build can swap them in:
//   neon_b200::computational_error       ~ neon::computational_error   (src/exceptions.hpp:14-17)
//   neon_b200::conjugate_gradient        ~ neon::conjugate_gradient    (linear_solver.hpp:59-71,
//                                           linear_solver.cpp:67-109): solve(A, x, b) on a CSR
//   neon_b200::solid_mesh                ~ mechanics::solid::mesh<submesh> (mesh.hpp:21-123):
//                                           update_internal_variables, save_internal_variables
//   neon_b200::static_matrix             ~ mechanics::static_matrix    (static_matrix.hpp:29-107):
//                                           construct, then solve()
// Recoverable numerical failures throw computational_error (static_matrix's cutback is inside
// nb2_static_solve); bad input throws std::domain_error; CUDA failures throw std::runtime_error.
#pragma once

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "neon_b200.h"

namespace neon_b200 {

class computational_error : public std::runtime_error {
public:
    computational_error(int status, std::string const& what)
        : std::runtime_error(what), status_(status) {}
    int status() const noexcept { return status_; }

private:
    int status_;
};

inline std::string last_error(nb2_ctx const* ctx) {
    char buf[512];
    nb2_last_error(ctx, buf, sizeof buf);
    return buf;
}

inline void check(int status, nb2_ctx const* ctx, char const* what) {
    if (status == NB2_OK) return;
    std::string msg = std::string(what) + ": " + last_error(ctx);
    switch (status) {
        case NB2_E_INPUT: throw std::domain_error(msg);
        case NB2_E_CUDA:
        case NB2_E_TIMEOUT: throw std::runtime_error(msg);
        default: throw computational_error(status, msg);
    }
}

/// Jacobi-preconditioned CG on the device for a CSR matrix (row pointer, column index, value)
/// as neon's Eigen RowMajor sparse_matrix stores it (outerIndexPtr, innerIndexPtr, valuePtr).
class conjugate_gradient {
public:
    explicit conjugate_gradient(double residual_tolerance = 1.0e-5,
                                std::int32_t max_iterations = 2000)
        : residual_tolerance(residual_tolerance), max_iterations(max_iterations) {}

    void solve(std::int32_t rows, std::int32_t const* row_ptr, std::int32_t const* col_idx,
               double const* values, std::vector<double>& x, std::vector<double> const& b) {
        x.assign(static_cast<std::size_t>(rows), 0.0);
        int st = nb2_pcg_solve(rows, row_ptr, col_idx, values, b.data(), x.data(),
                               residual_tolerance, max_iterations, &iterations_, &error_);
        if (st == NB2_E_CG_MAXIT)
            throw computational_error(st, "Conjugate gradient solver maximum iterations reached");
        if (st == NB2_E_NAN) throw computational_error(st, "Floating point error reported\n");
        check(st, nullptr, "conjugate_gradient");
    }

    std::int32_t iterations() const noexcept { return iterations_; }
    double error() const noexcept { return error_; }

private:
    double residual_tolerance;
    std::int32_t max_iterations;
    std::int32_t iterations_ = 0;
    double error_ = 0.0;
};

/// Device-resident mesh: coordinates, connectivity, CSR pattern, quadrature-point state.
class solid_mesh {
public:
    solid_mesh(std::vector<double> coordinates, std::vector<std::int32_t> connectivity,
               std::int32_t nodes_per_element, nb2_material const& material)
        : X(std::move(coordinates)), conn(std::move(connectivity)) {
        nb2_mesh_desc d{static_cast<std::int32_t>(X.size() / 3), X.data(),
                        static_cast<std::int32_t>(conn.size() / nodes_per_element),
                        nodes_per_element, conn.data()};
        check(nb2_create(&d, &material, &ctx), nullptr, "nb2_create");
        check(nb2_get_sizes(ctx, &dofs, &nnz, nullptr), ctx, "nb2_get_sizes");
    }
    solid_mesh(solid_mesh const&) = delete;
    solid_mesh& operator=(solid_mesh const&) = delete;
    ~solid_mesh() { nb2_destroy(ctx); }

    std::int32_t active_dofs() const noexcept { return dofs; }
    std::int64_t non_zeros() const noexcept { return nnz; }

    void update_internal_variables(std::vector<double> const& u, double dt = 0.0) {
        check(nb2_update_internal_variables(ctx, u.data(), dt), ctx, "update_internal_variables");
    }
    void save_internal_variables(bool have_converged) {
        check(nb2_save_internal_variables(ctx, have_converged ? 1 : 0), ctx,
              "save_internal_variables");
    }
    /// CSR pattern (row pointer, column index) exactly as compute_sparsity_pattern builds it
    std::pair<std::vector<std::int32_t>, std::vector<std::int32_t>> sparsity_pattern() const {
        std::vector<std::int32_t> rp(dofs + 1), col(nnz);
        check(nb2_export_pattern(ctx, rp.data(), col.data()), ctx, "export_pattern");
        return {rp, col};
    }
    /// tangent stiffness (CSR values) and internal force of the last update
    void assemble(std::vector<double>& K, std::vector<double>& f_int) {
        K.resize(static_cast<std::size_t>(nnz));
        f_int.resize(static_cast<std::size_t>(dofs));
        check(nb2_assemble(ctx, K.data(), f_int.data()), ctx, "assemble");
    }
    nb2_ctx* handle() noexcept { return ctx; }

private:
    std::vector<double> X;
    std::vector<std::int32_t> conn;
    nb2_ctx* ctx = nullptr;
    std::int32_t dofs = 0;
    std::int64_t nnz = 0;
};

/// A Dirichlet boundary or nodal force: DOFs plus a time/value table.
struct dof_table {
    std::vector<std::int32_t> dofs;
    std::vector<double> times, values, weights;
};

class mesh;  // a part read from neon's deck and .mesh file (neon_b200_json.hpp)

/// How a deck that asks for a direct linear solver ("direct", "PaStiX", "MUMPS") is solved:
/// refused (the default), or by the PCG at the given settings.
struct direct_solver_substitute {
    bool allowed = false;
    double tolerance = 1.0e-10;
    std::int32_t maximum_iterations = 20000;
};

/// Full-Newton quasi-static solver with adaptive load stepping.
class static_matrix {
public:
    static_matrix(solid_mesh& mesh, nb2_solver_options const& options,
                  std::vector<dof_table> dirichlet, std::vector<dof_table> nodal_forces = {})
        : mesh(mesh), options(options), dirichlet(std::move(dirichlet)),
          forces(std::move(nodal_forces)) {}

    /// static_matrix(mesh_type&, json const& simulation) (static_matrix.hpp:109-143): the
    /// options from the step's "nonlinear_options", "time" and "linear_solver"; the boundaries
    /// from the part.  Defined in neon_b200_json.hpp.
    template <class Json>
    static_matrix(::neon_b200::mesh& part, Json const& simulation,
                  std::int32_t precision = NB2_FP64,
                  direct_solver_substitute const& direct = direct_solver_substitute{});

    void solve() {
        auto pack = [](std::vector<dof_table> const& in) {
            std::vector<nb2_dof_table> out;
            for (auto const& t : in)
                out.push_back({t.dofs.data(), static_cast<std::int32_t>(t.dofs.size()),
                               t.times.data(), t.values.data(),
                               static_cast<std::int32_t>(t.times.size()),
                               t.weights.empty() ? nullptr : t.weights.data()});
            return out;
        };
        auto d = pack(dirichlet);
        auto f = pack(forces);
        u.assign(static_cast<std::size_t>(mesh.active_dofs()), 0.0);
        log.resize(100000);
        int st = nb2_static_solve(mesh.handle(), &options, d.data(), static_cast<int>(d.size()),
                                  f.data(), static_cast<int>(f.size()), u.data(), &report_,
                                  log.data(), static_cast<int>(log.size()));
        log.resize(static_cast<std::size_t>(std::min<std::int64_t>(report_.newton_iterations,
                                                                   100000)));
        if (st == NB2_E_CUTBACK_LIMIT) throw std::domain_error(report_.message);
        check(st, mesh.handle(), "static_matrix::solve");
    }

    std::vector<double> const& displacement() const noexcept { return u; }
    nb2_solve_report const& report() const noexcept { return report_; }
    std::vector<nb2_newton_log> const& newton_log() const noexcept { return log; }

private:
    solid_mesh& mesh;
    nb2_solver_options options;
    std::vector<dof_table> dirichlet, forces;
    std::vector<double> u;
    nb2_solve_report report_{};
    std::vector<nb2_newton_log> log;
};

}  // namespace neon_b200
