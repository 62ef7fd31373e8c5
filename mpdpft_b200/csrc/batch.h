// batch.h -- many independent SC solves advanced together (host side).
//
// The solves of a batch share their kernel instantiations (dimension 2,
// species count, precision, density functional, Pulay window) and may have
// different grid sizes.  fft.cu provides the batched transforms and the V
// assembly; batch.cu the SC kernels, the graph and the C ABI.
#pragma once
#include <vector>

#include "engine.h"

namespace mpdpft {

// One member of a batch: its context and its index in the batch.
struct BatchMember {
  Ctx* c;
  int index;
};

// DelField (method 5) of every species of the members whose grid size is
// the same, as six batched launches; vmax_all[index * kMaxS + s] is the
// taper shift of species s of a member.
struct BatchFftClass;
int batch_fft_create(const std::vector<BatchMember>& members, unsigned long long* vmax_all, BatchFftClass** out);
int batch_fft_issue(BatchFftClass* b, cudaStream_t st);
// the Coulomb terms of every argument set of the class (2D kernel, into each
// member's vh), when its solves have Coulomb interactions
bool batch_fft_has_coulomb(const BatchFftClass* b);
int batch_fft_issue_coulomb(BatchFftClass* b, cudaStream_t st);
void batch_fft_destroy(BatchFftClass* b);

// Rows of V-residual partial sums the V assembly of c writes.
double* batch_vres_part(const Ctx& c);

// The V assembly of every member in one launch (update 1), or the taper
// shell maxima of the current V only (update 0).  *blocks_out[k] is the
// number of V-residual partial rows member k's assembly writes.
struct BatchAssemble;
int batch_assemble_create(const std::vector<BatchMember>& members, unsigned long long* vmax_all,
                          BatchAssemble** out, std::vector<int>* blocks_out);
int batch_assemble_issue(BatchAssemble* b, int update, cudaStream_t st);
void batch_assemble_destroy(BatchAssemble* b);

}  // namespace mpdpft
