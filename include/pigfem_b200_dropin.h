/*
 * pigfem_b200_dropin.h -- binding calls of the drop-in Assembler::assemble
 * (pigfem_b200/drop_in/Assembler_b200.cpp).
 *
 * That translation unit replaces the reference's src/Assembler.cpp definition of
 *     PetscErrorCode Assembler::assemble(pmatrix& K, pvector& P_int, double delta_t,
 *                                        std::vector<std::vector<std::vector<double>>>& update_ISVs,
 *                                        NodalData* solution, bool assembleFunc, bool assembleJac)
 * (include/Assembler.h:46-48, src/Assembler.cpp:65-146) inside the reference's own build; every
 * solver keeps calling it as before (SolverNonlinearKSP.cpp:62,70,104; SolverLinear.cpp:66-71).
 * The reference's Problem is set up as usual (Problem::init / Problem::setup); the calls below
 * attach a B200 context to it.  The context is described by the same pg_problem_desc the C ABI
 * takes (the structured mesh, inclusions, materials, cohesive law and loading the driver gave the
 * reference's Mesh / Problem / BoundaryObject, Tests/Main.cpp:150-648), so its DOF numbering and
 * CSR patterns are the reference's own.  Serial (SeqAIJ) matrices only.
 */
#ifndef PIGFEM_B200_DROPIN_H_
#define PIGFEM_B200_DROPIN_H_

#include "pigfem_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Attach a B200 context built from desc to the reference Problem* `problem` (pg_create); every
 * later Assembler::assemble of that problem runs on the device.  Returns PG_OK or a PG_ERR_*
 * code (the message from pg_dropin_last_error).  Binding a problem again replaces its context. */
int pg_dropin_bind(void* problem, const pg_problem_desc* desc);
/* Detach and destroy the context of `problem` (no-op if none). */
int pg_dropin_unbind(void* problem);
/* Message of the last failed bind or assembly in this process. */
const char* pg_dropin_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* PIGFEM_B200_DROPIN_H_ */
