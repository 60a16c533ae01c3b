/*
 * pdlpgpu_mps.h -- MPS files in and out, fast.
 *
 * The reader replaces mps::MpsReader::read (include/mps/mps_reader.h:58-70,
 * src/mps/mps_reader.cpp:87-443): same sections and records (NAME, OBJSENSE,
 * ROWS, COLUMNS with INTORG/INTEND markers, RHS with an optional set name and
 * the objective constant, RANGES, BOUNDS LO UP FX FR MI PL BV LI UI,
 * QUADOBJ, QMATRIX, ENDATA), the same refusals (SOS, INDICATORS, QCMATRIX,
 * QCROWS, unknown headers, senses and bound types) with the same messages,
 * the same warnings, and the same model: variables in order of first
 * appearance with their names, types and bounds (the negative-UP rule
 * included), rows with their names and final bounds (RANGES applied as the
 * reference does), the objective constant, and per row the set of terms
 * with duplicate (row, column) pairs summed in file order and explicit zeros
 * kept. Terms are listed by increasing column index (the reference lists them
 * in hash-map order, which carries no meaning).
 *
 * It reads the whole file once and resolves names through one hash table per
 * kind, where the reference keeps a string map per term.
 *
 * pdlpgpu_mps_lp restates adapter::toCompiledLp (src/adapter/pdlp_adapter.cpp:
 * 21-189) so a file can go to the engine without the reference's pipeline.
 */
#ifndef PDLPGPU_MPS_H
#define PDLPGPU_MPS_H

#include <stdint.h>

#include "pdlpgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pdlpgpu_mps pdlpgpu_mps;

/* Reads an MPS file. Returns 0 and a model to release with pdlpgpu_mps_free,
 * or -1 with pdlpgpu_last_error() holding the reference reader's message
 * ("MpsReader Error (line N): ..."). */
int32_t pdlpgpu_mps_read(const char* path, pdlpgpu_mps** model);
void pdlpgpu_mps_free(pdlpgpu_mps* model);

/* sizes[8] = {variables, constraints, objective terms, constraint terms,
 * quadratic terms, warnings, sense (0 minimize, 1 maximize), integer or binary
 * variables}. */
void pdlpgpu_mps_sizes(const pdlpgpu_mps* model, int64_t* sizes);

/* Names: kind 0 the model name (index ignored), 1 variable `index`, 2 row
 * `index`, 3 warning `index`. The string lives as long as the model; NULL for
 * an index out of range. */
const char* pdlpgpu_mps_name(const pdlpgpu_mps* model, int32_t kind, int64_t index);

/* The model's arrays (sizes from pdlpgpu_mps_sizes; any pointer may be NULL to
 * skip it): objective constant; objective terms (variable, value); per
 * variable its type (0 continuous, 1 integer, 2 binary, model::VariableType)
 * and bounds; per row its bounds and terms as CSR (row_start[constraints + 1],
 * row_index / row_value); quadratic terms (i <= j, value) as
 * model::QuadraticTerm carries them. */
void pdlpgpu_mps_model(const pdlpgpu_mps* model, double* objective_offset,
                       int32_t* objective_index, double* objective_value, int32_t* var_type,
                       double* var_lower, double* var_upper, double* row_lower,
                       double* row_upper, int64_t* row_start, int32_t* row_index,
                       double* row_value, int32_t* quadratic_i, int32_t* quadratic_j,
                       double* quadratic_value);

/* adapter::toCompiledLp of the model: the LP the engine solves (minimisation;
 * a maximisation model has its objective and constant negated and
 * *objective_negated set). `lp` points into arrays the model owns, valid until
 * pdlpgpu_mps_free. Returns 0, or -1 with the adapter's message (quadratic or
 * integer models, bounds out of order, non-finite coefficients). */
int32_t pdlpgpu_mps_lp(pdlpgpu_mps* model, pdlpgpu_lp* lp, int32_t* objective_negated);

/* Writes `lp` as free-format MPS that pdlpgpu_mps_read and the reference
 * reader read back to the same LP bit for bit (17 significant digits): rows
 * with equal bounds as E, one-sided rows as L or G, two-sided rows as G with a
 * RANGES entry; variables and rows named x<j> and r<i>. Rows with no finite
 * bound cannot be written (an N row is dropped by readers) and give -1. */
int32_t pdlpgpu_mps_write(const char* path, const pdlpgpu_lp* lp, const char* name);

#ifdef __cplusplus
}
#endif

#endif /* PDLPGPU_MPS_H */
