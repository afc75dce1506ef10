/* CPU oracle for the cudaRing hot path: a plain-C restatement of the
 * reference algorithm (farceri/cudaRing), used ONLY as the checker by tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg.  Nothing in the
 * shipped library links or calls it.
 *
 * Parity of this restatement is pinned against the reference's own kernels
 * compiled as host code (oracle/_ref, built by oracle/build_ref.sh) through
 * the golden fixtures in tests/golden/.
 *
 * Layout follows the reference: positions/velocities/forces AoS
 * [x0,y0,x1,y1,...] float64, ring-contiguous vertex order, int64 indices,
 * neighbour list row-major [Nv x listSize] padded with -1.
 */
#ifndef CR_ORACLE_H
#define CR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OC_HARMONIC = 0, OC_LJ = 1, OC_ADHESIVE = 2, OC_WCA = 3 };
enum { OC_VERTEX_VERTEX = 0, OC_VERTEX_SMOOTH = 1, OC_CELL_SMOOTH = 2, OC_ALL = 3 };
enum { OC_MONO_HARMONIC = 0, OC_MONO_FENE = 1 };

typedef struct {
  long np, nv;
  const long* nv_list;   /* [np] */
  const long* first;     /* [np] */
  const long* pid;       /* [nv] */
  double lx, ly;
  double ea, el, eb, ec, l1, l2;
  double lj_cutoff, lj_ecut, lj_fshift, stiff, ext_sq;
  int potential, interaction, monomer;
} oc_sys;

/* include/cudaKernel.cuh:1571-1606 */
void oc_particle_shape(const oc_sys* s, const double* pos, double* length, double* theta,
                       double* area, double* perimeter);
/* include/cudaKernel.cuh:365-388, 1608-1613 */
void oc_particle_positions(const oc_sys* s, const double* pos, double* ppos);
/* include/cudaKernel.cuh:474-529 */
void oc_shape_force_energy(const oc_sys* s, const double* a0, const double* area, const double* ppos,
                           const double* l0, const double* theta0, const double* theta,
                           const double* pos, double* force, double* energy);
/* include/cudaKernel.cuh:690-722 */
void oc_vertex_interaction(const oc_sys* s, const double* rad, const double* pos, const long* nbr,
                           const long* cnt, long list_size, double* force, double* energy);
/* include/cudaKernel.cuh:725-757 */
void oc_all_to_all_interaction(const oc_sys* s, const double* rad, const double* pos, double* force,
                               double* energy);
/* include/cudaKernel.cuh:922-975 */
void oc_smooth_interaction(const oc_sys* s, const double* rad, const double* pos, const long* nbr,
                           const long* cnt, long list_size, double* force, double* p_energy);
/* include/cudaKernel.cuh:1735-1763: fills rows up to list_size, writes the
 * per-vertex count and returns the maximum count. */
long oc_neighbor_list(const oc_sys* s, const double* pos, const double* rad, double cut_distance,
                      long list_size, long* nbr, long* cnt);
/* include/cudaKernel.cuh:1906-1914 reduced: 1 when any vertex moved more than cutoff/3 */
int oc_check_displacement(const oc_sys* s, const double* pos, const double* last_pos, double cutoff);
/* DPM2D::calcForceEnergyGPU for periodic geometry (src/DPM2D.cu:1976-1993, 2058-2104);
 * scratch arrays: length, theta [nv], area, perimeter [np], ppos [2 np]. */
void oc_calc_force_energy(const oc_sys* s, const double* pos, const double* rad, const double* a0,
                          const double* l0, const double* theta0, const long* nbr, const long* cnt,
                          long list_size, double* force, double* energy, double* p_energy,
                          double* length, double* theta, double* area, double* perimeter, double* ppos);

/* Rigid path (include/cudaKernel.cuh:1412-1492). */
void oc_rigid_force_energy(const oc_sys* s, const double* pos, const double* rad, const long* nbr,
                           const long* cnt, long list_size, double* ppos, double* force,
                           double* torque, double* energy, double* moi, double* p_force,
                           double* p_torque, double* p_energy);
/* include/cudaKernel.cuh:1678-1713 */
void oc_translate_rotate(const oc_sys* s, const double* ppos, const double* plast_pos,
                         const double* pangle, const double* plast_angle, double* pos);

/* Philox4x32-10 counter-based generator (Salmon et al., SC'11) and the
 * Box-Muller normal pair used by the library's stochastic integrators. */
void oc_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void oc_normal2(uint64_t seed, uint64_t stream, uint64_t index, double out[2]);

#ifdef __cplusplus
}
#endif
#endif
