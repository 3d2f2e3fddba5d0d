/* C ABI of the batched solver (B200, sm_100a): many independent sheets of
 * uneven size stepped together. No counterpart in the reference, which steps
 * one scene per ClothSolver; each sheet here follows the reference's step
 * (src/solver/newton.ts:27-303) with floor contact
 * (src/collision/contact-assembly.ts, kind 2), in mixed precision (FP32
 * Jacobi-PCG, FP64 gradients, energies, dot products and floor CCD).
 *
 * Packing: sheets s = 0..S-1 each come with their own cs_mesh (local vertex
 * ids), cs_material and pins; positions and velocities are packed sheet after
 * sheet (3 doubles per vertex). pin_counts[s] pins of sheet s take the next
 * pin_counts[s] entries of pin_ids (local ids) and pin_pos (3 doubles each).
 *
 * One step is ONE persistent kernel launch: each thread block takes a sheet
 * from a work list ordered largest first and runs that sheet's whole implicit
 * step with block barriers only. cs_batch_step with steps > 1 captures the
 * sequence once into a CUDA graph and replays it. cs_batch_autotune times the
 * candidate launch shapes (128, 256 or 512 threads per block, i.e. vertices
 * per thread of a sheet; all resident blocks or a half or a third of them,
 * i.e. sheets in flight per SM) on the batch's own state (restored
 * afterwards) and keeps the fastest: fewer blocks keep fewer sheets in flight,
 * whose working sets then stay in L2.
 */
#ifndef CLOSIM_BATCH_H
#define CLOSIM_BATCH_H

#include <stdint.h>

#include "closim_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cs_batch cs_batch;

/* Per-sheet results of the last step, 8 doubles per sheet: Newton iterations,
 * PCG iterations, final gradient norm, energy, converged (1, or -1 for a
 * non-finite gradient), Armijo trials, active floor contacts, rejected trials. */
enum { CS_BATCH_STATS = 8 };

cs_batch* cs_batch_create(int32_t device);  /* NULL if the device does not exist */
void cs_batch_destroy(cs_batch* b);
const char* cs_batch_last_error(cs_batch* b);
int cs_batch_initialize(cs_batch* b, int32_t sheets, const cs_mesh* meshes, const cs_material* mats,
                        const double* x, const double* v, const int32_t* pin_counts, const int32_t* pin_ids,
                        const double* pin_pos, const double* gravity);
/* Floor contact (barrier, lagged friction, floor CCD) for every sheet. */
int cs_batch_set_contact(cs_batch* b, const cs_contact_params* p, int32_t floor_on, double floor_y);
/* Newton / PCG / line-search budgets and gradTol; Jacobi preconditioner only. */
int cs_batch_set_stepper_options(cs_batch* b, const cs_stepper_options* o);
int cs_batch_step(cs_batch* b, double dt, int32_t steps);
int cs_batch_get_positions(cs_batch* b, double* out);
int cs_batch_get_velocities(cs_batch* b, double* out);
int cs_batch_stats(cs_batch* b, double* out);  /* CS_BATCH_STATS doubles per sheet */
int cs_batch_autotune(cs_batch* b, double dt, int32_t* threads);
int cs_batch_set_threads(cs_batch* b, int32_t threads);
/* The launch shape in use: threads per block and resident blocks. */
int cs_batch_launch_shape(cs_batch* b, int32_t* threads, int32_t* blocks);
void* cs_batch_stream(cs_batch* b);

#ifdef __cplusplus
}
#endif

#endif /* CLOSIM_BATCH_H */
