// neon_b200_json.hpp -- neon's input deck and .mesh file for the C++ adapter (include/neon_b200.hpp).
//
// Header-only and templated on the JSON type, so a neon build passes its own neon::json
// (nlohmann::json, src/io/json.hpp) values.  The functions keep neon's keys, defaults and
// std::domain_error messages:
//   neon_b200::basic_mesh             ~ neon::basic_mesh (basic_mesh.cpp:8-19,
//                                       nodal_coordinates.cpp:13-33) with gmsh ordering converted
//                                       (node_ordering_adapter.cpp:46-68)
//   neon_b200::make_constitutive_model ~ make_constitutive_model (constitutive_model_factory.cpp:
//                                       26-161) + isotropic_elastic_property (:10-43) for the
//                                       models on the path
//   neon_b200::make_solver_options    ~ static_matrix's nonlinear options (static_matrix.hpp:
//                                       109-143), adaptive_time_step::parse_input and
//                                       check_increment_data (adaptive_time_step.cpp:108-160),
//                                       make_linear_solver (linear_solver_factory.cpp:20-120)
//   neon_b200::describe_mesh          ~ mechanics::solid::mesh's constructor (mesh.cpp:24-143,
//                                       229-248): the part, its boundaries and non-follower loads
//   neon_b200::mesh                   the description plus its device context
//   neon_b200::static_matrix(mesh&, simulation)   ~ static_matrix(mesh_type&, json const&)
// A neon module builds them in its own order (solid_mechanics_module.cpp:9-17):
//   neon_b200::basic_mesh part(mesh_file);
//   neon_b200::mesh m(part, material, simulation["meshes"].front(),
//                     simulation["time"]["increments"]["initial"]);
//   neon_b200::static_matrix solver(m, simulation);
//   solver.solve();
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "neon_b200.hpp"

namespace neon_b200 {

/// One element group of a .mesh file in neon's local node order.
struct element_group {
    std::int32_t gmsh_type = 0;
    std::int32_t nodes_per_element = 0;
    std::vector<std::int32_t> connectivity;  // [elements][nodes_per_element]

    std::int64_t elements() const {
        return nodes_per_element ? std::int64_t(connectivity.size()) / nodes_per_element : 0;
    }
};

/// gmsh type -> nodes per element for the types on this path (mesh/element_topology.hpp:
/// 2 triangle3, 3 quadrilateral4, 4 tetrahedron4, 5 hexahedron8); 0 for any other type.
inline std::int32_t gmsh_nodes(std::int32_t type) {
    switch (type) {
        case 2: return 3;
        case 3: return 4;
        case 4: return 4;
        case 5: return 8;
        default: return 0;
    }
}

namespace detail {

template <class Json>
bool has(Json const& j, char const* key) {
    return j.find(key) != j.end();
}

template <class Json>
std::vector<double> doubles(Json const& j) {
    std::vector<double> out;
    if (j.is_array())
        for (auto const& v : j) out.push_back(v.template get<double>());
    else
        out.push_back(j.template get<double>());
    return out;
}

/// sorted unique nodes of a group list (unique_dof_allocator, dof_allocator.hpp:19-37)
inline std::vector<std::int32_t> unique_nodes(std::vector<element_group> const& groups) {
    std::vector<std::int32_t> nodes;
    for (auto const& g : groups) nodes.insert(nodes.end(), g.connectivity.begin(), g.connectivity.end());
    std::sort(nodes.begin(), nodes.end());
    nodes.erase(std::unique(nodes.begin(), nodes.end()), nodes.end());
    return nodes;
}

}  // namespace detail

/// The coordinates and named element groups of a .mesh file.
class basic_mesh {
public:
    template <class Json>
    explicit basic_mesh(Json const& mesh_file) {
        for (char const* key : {"Nodes", "Elements"})
            if (!detail::has(mesh_file, key))
                throw std::domain_error(std::string("The mesh file is missing the \"") + key +
                                        "\" field");
        for (auto const& xyz : mesh_file.at("Nodes").at(0).at("Coordinates")) {
            if (xyz.size() != 3)
                throw std::domain_error("\"Coordinates\" must be a list of [x, y, z] triples");
            for (int k = 0; k < 3; ++k) X.push_back(xyz.at(k).template get<double>());
        }
        std::int64_t const nodes = std::int64_t(X.size() / 3);
        for (auto const& group : mesh_file.at("Elements")) {
            element_group g;
            g.gmsh_type = group.at("Type").template get<std::int32_t>();
            g.nodes_per_element = gmsh_nodes(g.gmsh_type);
            auto const name = group.at("Name").template get<std::string>();
            if (g.nodes_per_element == 0)
                throw std::domain_error("gmsh element type " + std::to_string(g.gmsh_type) +
                                        " is not on this path (hexahedron8, tetrahedron4 and "
                                        "their faces are)");
            for (auto const& element : group.at("NodalConnectivity")) {
                if (std::int32_t(element.size()) != g.nodes_per_element)
                    throw std::domain_error("group \"" + name + "\": type " +
                                            std::to_string(g.gmsh_type) + " needs " +
                                            std::to_string(g.nodes_per_element) +
                                            " nodes per element");
                std::int32_t n[8];
                for (std::int32_t a = 0; a < g.nodes_per_element; ++a) {
                    n[a] = element.at(a).template get<std::int32_t>();
                    if (n[a] < 0 || n[a] >= nodes)
                        throw std::domain_error("group \"" + name +
                                                "\" refers to a node that does not exist");
                }
                if (g.gmsh_type == 4) {  // gmsh tetrahedron4 -> neon's local order (1, 2, 3, 0)
                    std::int32_t const first = n[0];
                    n[0] = n[1];
                    n[1] = n[2];
                    n[2] = n[3];
                    n[3] = first;
                }
                g.connectivity.insert(g.connectivity.end(), n, n + g.nodes_per_element);
            }
            groups[name].push_back(std::move(g));
        }
    }

    /// node-major xyz
    std::vector<double> const& coordinates() const noexcept { return X; }
    std::int32_t nodes() const noexcept { return std::int32_t(X.size() / 3); }

    /// basic_mesh::meshes: every group of that name
    std::vector<element_group> const& meshes(std::string const& name) const {
        auto const it = groups.find(name);
        if (it == groups.end())
            throw std::domain_error("The mesh name \"" + name +
                                    "\" does not exist in the mesh file");
        return it->second;
    }

    /// the groups of one name joined into one group (one element type per name on this path)
    element_group joined(std::string const& name) const {
        auto const& list = meshes(name);
        element_group out;
        out.gmsh_type = list.front().gmsh_type;
        out.nodes_per_element = list.front().nodes_per_element;
        for (auto const& g : list) {
            if (g.gmsh_type != out.gmsh_type)
                throw std::domain_error("group \"" + name +
                                        "\" mixes element types; one element type per group is "
                                        "on this path");
            out.connectivity.insert(out.connectivity.end(), g.connectivity.begin(),
                                    g.connectivity.end());
        }
        return out;
    }

private:
    std::vector<double> X;
    std::map<std::string, std::vector<element_group>> groups;
};

/// The device model for a "constitutive" object and the part's material.
template <class Json>
nb2_material make_constitutive_model(Json const& material, Json const& constitutive) {
    using detail::has;
    if (!has(constitutive, "name"))
        throw std::domain_error("Missing \"name\" in \"constitutive\"");
    auto const name = constitutive.at("name").template get<std::string>();

    nb2_material m{};
    std::string type, statistics;
    if (name == "microsphere") {
        if (!has(constitutive, "type"))
            throw std::domain_error(
                "Missing \"type\" as \"affine\" or \"nonaffine\" in microsphere model");
        if (!has(constitutive, "quadrature"))
            throw std::domain_error(
                "Missing \"quadrature\" as \"BO21\", \"BO33\" or \"FM900\" in microsphere model");
        auto const rule = constitutive.at("quadrature").template get<std::string>();
        if (rule != "BO21" && rule != "BO33" && rule != "FM900")
            throw std::domain_error("\"quadrature\" field must be \"BO21\", \"BO33\" or \"FM900\"");
        type = constitutive.at("type").template get<std::string>();
        if (type == "affine") {
            if (!has(constitutive, "statistics"))
                throw std::domain_error("Missing \"statistics\" as \"gaussian\" or \"langevin\" in "
                                        "the microsphere model");
            statistics = constitutive.at("statistics").template get<std::string>();
            if (statistics != "gaussian" && statistics != "langevin")
                throw std::domain_error("\"statistics\" for the microsphere model must be either "
                                        "\"gaussian\" or \"langevin\"");
        } else if (type != "nonaffine") {
            throw std::domain_error("microsphere model options are \"affine\" or \"nonaffine\"");
        }
        if (rule == "FM900" || (type == "affine" && statistics == "gaussian" &&
                                has(constitutive, "ageing")))
            throw std::domain_error("the microsphere models (affine Gaussian, affine Langevin, "
                                    "non-affine) are on this path with the BO21 and BO33 rules");
        m.unit_sphere_points = rule == "BO33" ? 33 : 21;
    }

    // isotropic_elastic_property (isotropic_elastic_property.cpp:10-43)
    if (has(material, "bulk_modulus") && has(material, "shear_modulus")) {
        m.bulk_modulus = material.at("bulk_modulus").template get<double>();
        m.shear_modulus = material.at("shear_modulus").template get<double>();
    } else if (has(material, "elastic_modulus") && has(material, "poissons_ratio")) {
        double const E = material.at("elastic_modulus").template get<double>();
        double const nu = material.at("poissons_ratio").template get<double>();
        if (nu >= 0.5)
            throw std::domain_error("\"poissons_ratio\" must be less than or equal to 0.5");
        m.bulk_modulus = E / (3.0 * (1.0 - 2.0 * nu));
        m.shear_modulus = E / (2.0 * (1.0 + nu));
    } else {
        throw std::domain_error("\"elastic_modulus\" and \"poissons_ratio\" or \"bulk_modulus\" "
                                "and \"shear_modulus\" need to be specified as material "
                                "properties");
    }

    if (name == "neohooke" || name == "compressible_neohooke") {
        m.model = NB2_NEOHOOKE;
    } else if (name == "isotropic_linear_elasticity") {
        m.model = NB2_ISOTROPIC_LINEAR_ELASTICITY;
    } else if (name == "J2_plasticity") {
        if (!has(constitutive, "finite_strain"))
            throw std::domain_error("\"small_strain_J2_plasticity\" must have a boolean value for "
                                    "\"finite_strain\"");
        if (constitutive.at("finite_strain").template get<bool>())
            throw std::domain_error("finite-strain J2 is not on this path");
        if (!has(material, "yield_stress"))
            throw std::domain_error("\"yield_stress\" was not specified in material properties");
        m.model = NB2_SMALL_STRAIN_J2_PLASTICITY;
        m.yield_stress = material.at("yield_stress").template get<double>();
        m.isotropic_hardening_modulus =
            has(material, "isotropic_hardening_modulus")
                ? material.at("isotropic_hardening_modulus").template get<double>()
                : 0.0;
    } else if (name == "microsphere") {
        if (!has(material, "segments_per_chain"))
            throw std::domain_error("segments_per_chain not specified in material data");
        m.segments_per_chain = material.at("segments_per_chain").template get<double>();
        if (type == "nonaffine") {
            if (!has(material, "nonaffine_stretch_parameter"))
                throw std::domain_error(
                    "\"nonaffine_stretch_parameter\" not specified in material data");
            m.model = NB2_NONAFFINE_MICROSPHERE;
            m.nonaffine_stretch_parameter =
                material.at("nonaffine_stretch_parameter").template get<double>();
        } else {
            m.model = statistics == "gaussian" ? NB2_GAUSSIAN_AFFINE_MICROSPHERE
                                               : NB2_LANGEVIN_AFFINE_MICROSPHERE;
        }
    } else {
        throw std::domain_error("The model name " + name + " is not recognised");
    }
    return m;
}

/// nb2_solver_options from one load step of a deck (its "nonlinear_options", "time" and
/// "linear_solver" objects).
template <class Json>
nb2_solver_options make_solver_options(Json const& simulation, std::int32_t precision = NB2_FP64,
                                       direct_solver_substitute const& direct = {}) {
    using detail::has;
    nb2_solver_options o{};
    if (!has(simulation, "nonlinear_options"))
        throw std::domain_error("displacement_tolerance not specified in nonlinear_options");
    auto const& nl = simulation.at("nonlinear_options");
    if (!has(nl, "displacement_tolerance"))
        throw std::domain_error("displacement_tolerance not specified in nonlinear_options");
    if (!has(nl, "residual_tolerance"))
        throw std::domain_error("residual_tolerance not specified in nonlinear_options");
    o.residual_tolerance = nl.at("residual_tolerance").template get<double>();
    o.displacement_tolerance = nl.at("displacement_tolerance").template get<double>();
    o.linear_iterations =
        has(nl, "linear_iterations") ? nl.at("linear_iterations").template get<std::int32_t>() : 10;
    o.absolute_tolerance = has(nl, "absolute_tolerance") ? 1 : 0;

    if (!has(simulation, "time")) throw std::domain_error("A simulation case needs a \"time\" field");
    auto const& time = simulation.at("time");
    if (!has(time, "period")) throw std::domain_error("Time data requires a \"period\" value\n");
    if (!has(time, "increments")) throw std::domain_error("\"increments\" not provided!\n");
    auto const& inc = time.at("increments");
    if (!has(inc, "initial")) throw std::domain_error("increment initial value not provided!\n");
    if (!has(inc, "minimum")) throw std::domain_error("increment minimum value not provided!\n");
    if (!has(inc, "maximum")) throw std::domain_error("increment maximum value not provided!\n");
    if (!has(inc, "adaptive"))
        throw std::domain_error("\"adaptive\" (true or false) not provided in \"increments\"");
    o.adaptive = inc.at("adaptive").template get<bool>() ? 1 : 0;
    o.period = time.at("period").template get<double>();
    o.initial_increment = inc.at("initial").template get<double>();
    o.minimum_increment = o.adaptive ? inc.at("minimum").template get<double>() : o.initial_increment;
    o.maximum_increment = o.adaptive ? inc.at("maximum").template get<double>() : o.initial_increment;

    if (!has(simulation, "linear_solver") || !has(simulation.at("linear_solver"), "type"))
        throw std::domain_error("A \"linear_solver\" \"type\" must be specified");
    auto const& ls = simulation.at("linear_solver");
    auto const kind = ls.at("type").template get<std::string>();
    if (kind != "PaStiX" && kind != "MUMPS" && kind != "direct" && kind != "iterative")
        throw std::domain_error("Linear solver " + kind +
                                " is not recognised.  Please use \"PaStiX\", \"MUMPS\", "
                                "\"direct\" or \"iterative\"");
    if (kind == "iterative") {
        o.cg_tolerance = has(ls, "tolerance") ? ls.at("tolerance").template get<double>() : 1.0e-5;
        o.cg_maximum_iterations = has(ls, "maximum_iterations")
                                      ? ls.at("maximum_iterations").template get<std::int32_t>()
                                      : 2000;
    } else if (direct.allowed) {
        o.cg_tolerance = direct.tolerance;
        o.cg_maximum_iterations = direct.maximum_iterations;
    } else {
        throw std::domain_error("linear solver \"" + kind +
                                "\": the path solves with the Jacobi PCG (\"type\": "
                                "\"iterative\")");
    }
    o.precision = precision;
    o.mixed_inner_tolerance = 1.0e-2;
    o.use_graphs = 1;
    return o;
}

/// boundary::generate_sinusoidal (mesh/boundary/boundary.cpp:87-147): starts at (0, 0), then one
/// block of floor(cycles * period / generate_time_step) samples per entry, each block spread
/// evenly over its cycles and starting where the previous one ended.
inline std::pair<std::vector<double>, std::vector<double>> sinusoidal_table(
    std::vector<double> const& amplitude, std::vector<double> const& period,
    std::vector<double> const& number_of_cycles, std::vector<double> const& phase,
    double generate_time_step) {
    if (amplitude.size() != period.size() || period.size() != phase.size() ||
        phase.size() != number_of_cycles.size())
        throw std::domain_error("The amplitude, period, number_of_cycles, time_step and phase "
                                "vectors must be of the same size.");
    double const two_pi = 6.283185307179586476925286766559;
    std::vector<double> times{0.0}, values{0.0};
    for (std::size_t i = 0; i < amplitude.size(); ++i) {
        double const omega = two_pi / period[i];
        auto const steps =
            static_cast<std::int64_t>(number_of_cycles[i] * period[i] / generate_time_step);
        double const scale = number_of_cycles[i] * period[i] / double(steps);
        double const start = times.back();
        for (std::int64_t s = 1; s <= steps; ++s) {
            double const t = double(s) * scale + start;
            times.push_back(t);
            values.push_back(amplitude[i] * std::sin(omega * t + phase[i]));
        }
    }
    return {times, values};
}

/// boundary::allocate_time_load (boundary.cpp:150-176)
inline void check_time_table(std::vector<double> const& t, std::vector<double> const& v) {
    if (t.size() < 2) throw std::domain_error("\"time\" is not a vector of at least two elements");
    if (v.size() < 2)
        throw std::domain_error(
            "The specified boundary values do not contain at least two elements");
    if (t.size() != v.size())
        throw std::domain_error("The time and load vectors must be of the same size.");
    if (!std::is_sorted(t.begin(), t.end()))
        throw std::domain_error("Load times must be monotonically increasing.");
}

/// The time/value table of one component of a boundary (boundary.cpp:20-34).
template <class Json>
std::pair<std::vector<double>, std::vector<double>> boundary_table(Json const& boundary,
                                                                   char const* key,
                                                                   double generate_time_step) {
    using detail::has;
    std::pair<std::vector<double>, std::vector<double>> table;
    if (has(boundary, "generate_type")) {
        if (boundary.at("generate_type").template get<std::string>() != "sinusoidal")
            throw std::domain_error("\"generate_type\" must be \"sinusoidal\"");
        for (char const* field : {"period", "phase", "number_of_cycles"})
            if (!has(boundary, field))
                throw std::domain_error(std::string("\"") + field +
                                        "\" was not specified in \"boundaries\".");
        table = sinusoidal_table(detail::doubles(boundary.at(key)),
                                 detail::doubles(boundary.at("period")),
                                 detail::doubles(boundary.at("number_of_cycles")),
                                 detail::doubles(boundary.at("phase")), generate_time_step);
    } else {
        table = {detail::doubles(boundary.at("time")), detail::doubles(boundary.at(key))};
    }
    check_time_table(table.first, table.second);
    return table;
}

/// One non-follower load boundary: its kind (NB2_LOAD_*), component, faces and time table.
struct load_spec {
    std::int32_t kind = NB2_LOAD_TRACTION;
    std::int32_t component = 0;
    std::vector<std::int32_t> faces;  // [faces][nodes_per_face], surface loads
    std::int32_t nodes_per_face = 0;
    std::int32_t reduced_quadrature = 0;
    std::vector<double> times, values;
    std::string name;
};

/// Everything a part needs before it reaches the device: coordinates, connectivity, material,
/// Dirichlet tables (in static_matrix's order: names sorted, then x, y, z), nodal-force tables
/// and non-follower loads (deck order).
struct mesh_description {
    std::vector<double> coordinates;
    std::vector<std::int32_t> connectivity;
    std::int32_t nodes_per_element = 0;
    nb2_material material{};
    std::vector<dof_table> dirichlet;
    std::vector<dof_table> nodal_forces;
    std::vector<load_spec> loads;
};

/// mechanics::solid::mesh's constructor without the device: mesh_data is the step's
/// "meshes"[0] object, generate_time_step the step's initial increment.
template <class Json>
mesh_description describe_mesh(basic_mesh const& basic, Json const& material_data,
                               Json const& mesh_data, double generate_time_step) {
    using detail::has;
    mesh_description d;
    auto const part = mesh_data.at("name").template get<std::string>();
    if (!has(mesh_data, "constitutive"))
        throw std::domain_error("Missing \"constitutive\" in \"mesh\"");
    d.material = make_constitutive_model(material_data, mesh_data.at("constitutive"));

    element_group volume = basic.joined(part);
    if (volume.gmsh_type != 4 && volume.gmsh_type != 5)
        throw std::domain_error("part \"" + part + "\" is not a volume mesh");
    if (!has(mesh_data, "element_options"))
        throw std::domain_error("Missing \"part\": {\"element_options\" : {}}");
    auto const& eo = mesh_data.at("element_options");
    bool const reduced = has(eo, "quadrature") && eo.at("quadrature").is_string() &&
                         eo.at("quadrature").template get<std::string>() == "reduced";
    if (reduced && volume.gmsh_type == 5)
        throw std::domain_error("reduced (one-point) hexahedron8 quadrature is not on this path; "
                                "the element kernels integrate hexahedron8 with eight points");
    d.coordinates = basic.coordinates();
    d.connectivity = std::move(volume.connectivity);
    d.nodes_per_element = volume.nodes_per_element;

    static char const* const keys[3] = {"x", "y", "z"};
    std::map<std::string, std::vector<dof_table>> displacement;
    if (!has(mesh_data, "boundaries")) return d;
    auto const& boundaries = mesh_data.at("boundaries");
    for (auto const& b : boundaries) {  // check_boundary_conditions (mesh.cpp:229-248)
        for (char const* field : {"name", "type"})
            if (!has(b, field))
                throw std::domain_error(std::string("\"") + field +
                                        "\" was not specified in \"boundary\".");
        if (!has(b, "time") && !has(b, "generate_type"))
            throw std::domain_error(
                "Neither \"time\" nor \"generate_type\" was specified in \"boundary\".");
    }
    for (auto const& b : boundaries) {  // allocate_boundary_conditions (mesh.cpp:75-104)
        auto const name = b.at("name").template get<std::string>();
        auto const type = b.at("type").template get<std::string>();
        if (type == "displacement" || type == "nodal_force") {
            auto const nodes = detail::unique_nodes(basic.meshes(name));
            for (int k = 0; k < 3; ++k) {
                if (!has(b, keys[k])) continue;
                dof_table t;
                for (auto n : nodes) t.dofs.push_back(3 * n + k);
                std::tie(t.times, t.values) = boundary_table(b, keys[k], generate_time_step);
                (type == "displacement" ? displacement[name] : d.nodal_forces)
                    .push_back(std::move(t));
            }
        } else if (type == "traction" || type == "pressure") {
            element_group faces = basic.joined(name);
            if (faces.gmsh_type != 2 && faces.gmsh_type != 3)
                throw std::domain_error("surface load \"" + name + "\" is not a group of faces");
            auto add = [&](std::int32_t kind, std::int32_t comp, std::vector<double> t,
                           std::vector<double> v) {
                load_spec s;
                s.kind = kind;
                s.component = comp;
                s.faces = faces.connectivity;
                s.nodes_per_face = faces.nodes_per_element;
                s.reduced_quadrature = reduced ? 1 : 0;
                s.times = std::move(t);
                s.values = std::move(v);
                s.name = name;
                d.loads.push_back(std::move(s));
            };
            if (type == "pressure") {
                if (!has(b, "value"))
                    throw std::domain_error(
                        "Pressure boundary condition must specify a \"value\" array");
                auto t = detail::doubles(b.at("time"));
                auto v = detail::doubles(b.at("value"));
                check_time_table(t, v);
                add(NB2_LOAD_PRESSURE, 0, std::move(t), std::move(v));
            } else {
                for (int k = 0; k < 3; ++k) {
                    if (!has(b, keys[k])) continue;
                    auto tv = boundary_table(b, keys[k], generate_time_step);
                    add(NB2_LOAD_TRACTION, k, std::move(tv.first), std::move(tv.second));
                }
            }
        } else if (type == "body_force") {
            if (name != part)
                throw std::domain_error("a body force acts on the part's own elements on this "
                                        "path; \"" + name + "\" is another group");
            for (int k = 0; k < 3; ++k) {
                if (!has(b, keys[k])) continue;
                load_spec s;
                s.kind = NB2_LOAD_BODY_FORCE;
                s.component = k;
                std::tie(s.times, s.values) = boundary_table(b, keys[k], generate_time_step);
                s.name = name;
                d.loads.push_back(std::move(s));
            }
        } else {
            throw std::domain_error("boundary \"" + type + "\" is not recognised");
        }
    }
    for (auto& [name, tables] : displacement)  // std::map: names sorted, each in x, y, z order
        for (auto& t : tables) d.dirichlet.push_back(std::move(t));
    return d;
}

/// mechanics::solid::mesh on the device: the described part in a solid_mesh context, with the
/// non-follower loads turned into weighted nodal-force tables (their nodal vectors per unit
/// load value computed on the device, nb2_nonfollower_load).
class mesh {
public:
    template <class Json>
    mesh(basic_mesh const& basic, Json const& material_data, Json const& mesh_data,
         double generate_time_step)
        : description(describe_mesh(basic, material_data, mesh_data, generate_time_step)) {
        device_mesh = std::make_unique<solid_mesh>(description.coordinates,
                                                   description.connectivity,
                                                   description.nodes_per_element,
                                                   description.material);
        forces = description.nodal_forces;
        std::int32_t const ndofs = device_mesh->active_dofs();
        std::vector<double> f(static_cast<std::size_t>(ndofs));
        for (auto const& s : description.loads) {
            bool const surface = s.kind != NB2_LOAD_BODY_FORCE;
            std::int32_t const num_faces =
                surface ? std::int32_t(s.faces.size() / s.nodes_per_face) : 0;
            check(nb2_nonfollower_load(device_mesh->handle(), s.kind, s.component,
                                       surface ? s.faces.data() : nullptr, num_faces,
                                       surface ? s.nodes_per_face : 0, s.reduced_quadrature,
                                       f.data()),
                  device_mesh->handle(), "nonfollower_load");
            // the table's DOFs: the loaded nodes, the loaded components, ascending
            std::vector<std::int32_t> nodes;
            if (surface) {
                element_group g;
                g.connectivity = s.faces;
                nodes = detail::unique_nodes({g});
            } else {
                for (std::int32_t n = 0; n < ndofs / 3; ++n) nodes.push_back(n);
            }
            dof_table t;
            for (auto n : nodes)
                for (int k = 0; k < 3; ++k)
                    if (s.kind == NB2_LOAD_PRESSURE || k == s.component) t.dofs.push_back(3 * n + k);
            for (auto dof : t.dofs) t.weights.push_back(f[static_cast<std::size_t>(dof)]);
            t.times = s.times;
            t.values = s.values;
            forces.push_back(std::move(t));
        }
    }

    solid_mesh& device() noexcept { return *device_mesh; }
    std::int32_t active_dofs() const noexcept { return device_mesh->active_dofs(); }
    mesh_description const& describe() const noexcept { return description; }
    std::vector<dof_table> const& dirichlet_boundaries() const noexcept {
        return description.dirichlet;
    }
    /// nodal forces first, then the non-follower loads in deck order
    std::vector<dof_table> const& external_forces() const noexcept { return forces; }

    void update_internal_variables(std::vector<double> const& u, double dt = 0.0) {
        device_mesh->update_internal_variables(u, dt);
    }
    void save_internal_variables(bool have_converged) {
        device_mesh->save_internal_variables(have_converged);
    }

private:
    mesh_description description;
    std::unique_ptr<solid_mesh> device_mesh;
    std::vector<dof_table> forces;
};

template <class Json>
static_matrix::static_matrix(::neon_b200::mesh& part, Json const& simulation,
                             std::int32_t precision, direct_solver_substitute const& direct)
    : static_matrix(part.device(), make_solver_options(simulation, precision, direct),
                    part.dirichlet_boundaries(), part.external_forces()) {}

}  // namespace neon_b200
