// Internal helpers shared by the host translation units: the thread-local
// last-error message behind fe_last_error(), and status helpers.
#pragma once
#include <cstdint>
#include <string>

namespace fe {

// Record a failure for fe_last_error() and return its status code.
int fe_fail(int status, const std::string& msg);
void fe_clear_error();

// Autotuner decisions per size class (autotune.cpp): the brick (FE_BRICK_*)
// and steps per graph launch measured fastest for lattices of this
// dimensionality, storage, collision, near-wall rule, porosity (0.05 bins)
// and site count (powers of two). False when the class was not tuned.
bool tune_lookup(int dim2, int storage, int mrt, int hbb, double porosity, int64_t sites, int* brick,
                 int* graph_steps);
void tune_store(int dim2, int storage, int mrt, int hbb, double porosity, int64_t sites, int brick, int graph_steps);

}  // namespace fe

using fe::fe_fail;
