// y-slab decomposition of one domain over ranks (internal).
//
// The reference decomposes its domain over MPI ranks and, wherever a
// stencil needs the neighbour's rows, exchanges the ghost rows
// (SrcOrig/shiftsx.f90:139-205 and its y and second-layer siblings,
// SrcOrig/sethalo.f90:485-505); the global minimum of the sedimentation
// sub-step is an allreduce (SrcOrig/chkfall.f90:88).  Here a context in
// slab mode (Grid::slaby) writes no y ghosts itself; at the same points of
// the step it asks its SlabLink to fill them from the neighbours (y is
// periodic over the ring of ranks: rank 0's southern neighbour is the last
// rank) and to reduce the sub-step word.
//
// Rows exchanged per field (ghost <- neighbour's interior), per level:
//   rows 0, 1                   <- southern rank's rows nj-3, nj-2
//   rows nj-1, nj  (scalar, u)  <- northern rank's rows 2, 3
//   rows nj, nj+1  (v faces)    <- northern rank's rows 3, 4
// the rows the periodic wrap fills on a single domain (bcycle.f90:159-225
// with the shift2nd.f90 second layer), so a slab run computes what the
// single domain computes, the shared v face of two slabs on both sides.
#pragma once
#include <cuda_runtime.h>

namespace cress {

struct Ctx;

struct SlabLink {
  int rank = 0, nranks = 1;
  virtual ~SlabLink() {}
  // Fill the y ghost rows of nf fields of this rank (stag: STAG_* per
  // field) from the neighbours, ordered on the context's stream after the
  // work that wrote the fields and before the work that follows.
  virtual int exchange(Ctx* c, int nf, float* const* fields, const int* stag) = 0;
  // The minimum over ranks of a device int32 word (in place).
  virtual int min_word(Ctx* c, int* word) = 0;
};

}  // namespace cress
