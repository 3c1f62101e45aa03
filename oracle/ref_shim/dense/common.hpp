// Minimal stand-in for LvArray's dense linear-algebra front end as the reference's SCF drivers call it
// (oracle reference build, test infrastructure): option and backend tags and an empty workspace.
// The solvers are in dense/eigenDecomposition.hpp.
#pragma once

#include "../Array.hpp"

namespace LvArray {
namespace dense {

enum class BuiltInBackends { LAPACK, MAGMA, MAGMA_GPU };
enum class SymmetricMatrixStorageType { UPPER_TRIANGULAR, LOWER_TRIANGULAR };

struct EigenDecompositionOptions {
  enum Type { EIGENVALUES, EIGENVALUES_AND_RIGHT_VECTORS, EIGENVALUES_AND_LEFT_VECTORS, EIGENVALUES_AND_LEFT_AND_RIGHT_VECTORS };
  enum Problem { Ax_eq_lambdaBx, ABx_eq_lambdax, BAx_eq_lambdax };
  EigenDecompositionOptions(Type t, Problem p = Ax_eq_lambdaBx) : type(t), problem(p) {}
  Type type;
  Problem problem;
};

template <typename T, template <typename> class BUFFER>
struct ArrayWorkspace {};

}  // namespace dense
}  // namespace LvArray
