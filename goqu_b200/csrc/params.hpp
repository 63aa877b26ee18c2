// Binding of goqu's parameterized gates from parameter values, on the host
// side of the engine, so that an optimisation loop rebinds a circuit without
// its caller rebuilding matrices (circuit/gate/parameterized.go:91-564,
// circuit/param/gate.go:13-142).
#pragma once
#include <stddef.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/gqb200.h"
#include "schedule.hpp"

namespace gq {

// Matrix of one gate family at the given angles (row major, first qubit MSB).
// Returns false for an unknown family or angle count.
bool param_gate_matrix(int family, const double* angles, int n_angles, std::vector<Z>& m);
// d(matrix)/d(angle k) of the family at the given angles.
bool param_gate_dmatrix(int family, const double* angles, int n_angles, int k, std::vector<Z>& dm);

// Binds the template: ops are copied; each gq_param_gate's op gets the
// family's matrix at its angles (angle k = scale[k] * theta[param[k]] + shift[k])
// and, per distinct parameter, d(matrix)/d(parameter) with the chain rule
// applied (param_index / dmatrix). `store` owns the matrices the copies point to.
struct BoundTemplate {
    std::vector<gq_op> ops;
    std::vector<std::vector<Z>> store;
};
int bind_template(const gq_op* ops, size_t n_ops, const gq_param_gate* pg, size_t n_pg, const double* theta,
                  size_t n_params, BoundTemplate& out, std::string& err);

}  // namespace gq
