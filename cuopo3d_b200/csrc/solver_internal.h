// Internal C++ interface between the single-instance solver (opo_host.cu) and the batch
// / serving layer (batch.cu).  Not part of the C-ABI.
#pragma once

#include "../../include/cuopo3d.h"
#include "opo_internal.h"

namespace opo {

// Device bytes a batch charges one instance against its HBM budget: the four fields
// (Api, Ap, As, Ai) of nx ny nt complex values plus 1 MiB for its plans and tables.
// The serving loop's admission uses the same count.
inline size_t batch_instance_bytes(int precision, size_t voxels)
{
    const size_t esz = precision == OPO_FP64 ? 16 : 8;
    return 4 * esz * voxels + ((size_t)1 << 20);
}

// Create a solver with the given kernel variant and tile size per pass (t, x, y);
// `stream` (may be null) replaces the solver's own stream, e.g. a batch's stream.
int solver_create_configured(const OpoParams *p, const double *w, const PassVariant v[3], const size_t te[3],
                             cudaStream_t stream, OpoSolver **out);
void solver_pass_info(const OpoSolver *s, int kind, int *ntiles, size_t *smem);
PassVariant solver_pass_variant(const OpoSolver *s, int kind);
// A line-specialised t-pass setting runs its line body on s's grid, or its generic
// fallback with the setting's fallback radix (what a batch's kernel compiles).
bool solver_line_fallback_ok(const OpoSolver *s);
// The line body's time axis the t-pass runs on s's grid (0: the generic body).
int solver_line_nt(const OpoSolver *s);
const OpoParams &solver_params(const OpoSolver *s);
size_t solver_device_bytes(const OpoSolver *s);
void *solver_field(OpoSolver *s, int which);
bool solver_gdd_or_mirror(const OpoSolver *s);
// z of the half steps of t-pass number tp of a round trip (tp = 0 .. n_steps) and how
// many half steps that pass takes.
void solver_tpass_z(const OpoParams &p, int tp, double zh[2], int *n_rk4);
// Frees the solver's precision-conversion buffer, if any (it is re-created on demand).
void solver_release_staging(OpoSolver *s);
// Sets the last error string of a solver (for errors found by the batch layer).
int solver_fail(OpoSolver *s, int code, const char *msg);

cudaStream_t solver_stream(const OpoSolver *s);
// Device initialisation of Api, Ap (pump), As (seeded noise), Ai (zero or As) (init_fields.cu).
int init_fields_device(OpoSolver *s, const OpoConfig *cfg, unsigned long long seed, double sigma, int idler_copy,
                       cudaStream_t stream);

template <typename C>
TPassArgs<C> make_tpass_args(OpoSolver *s, bool reset_pump, int n_rk4, const double *zh, int which_tab,
                             unsigned tmask);
template <typename C> AxisArgs<C> make_axis_args(OpoSolver *s, int kind, int which_tab, unsigned mask);

}  // namespace opo
