// scc_compat.h -- the reference's own entry points, provided by
// libscc_b200.so with the reference's exact C++ signatures (and so the same
// mangled names), so that code written against the reference links
// unchanged.
//
//   reference declaration                         mangled name
//   scc.h:52  vHong(...)                           _Z5vHongjjPjS_S_S_bb
//   scc.h:50  vSlota(...)                          _Z6vSlotajjPjS_S_S_bb
//   scc.h:51  wHong(..., int warpSize)             _Z5wHongjjPjS_S_S_bbi
//   scc.h:49  wSlota(..., int warpSize)            _Z6wSlotajjPjS_S_S_bbi
//   load.h:6  loadFullGraph(...)                   _Z13loadFullGraphPKcPjS1_PS1_S2_S2_S2_S2_
//   scc.h:53  detectSCC(...) (stub: throws)         _Z9detectSCCjjPjS_S_S_S_bb
//
// Behaviour kept from the reference: the drivers return nothing and print
// "[numberOf1Sccs: N\n]\nNumber Of Sccs : N\nTime : T" (scc_WCC.cu:948-967,
// scc_Coloring.cu:669-670); running out of device memory throws the
// reference's const char* message (scc_WCC.cu:618-623); any other CUDA
// failure prints a GPUassert line and exits with the error code
// (scc.h:12-20).  RSize is V and CSize is E.
#ifndef SCC_COMPAT_H
#define SCC_COMPAT_H

#include <stdint.h>

void vHong(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, bool t1, bool t2);
void vSlota(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, bool t1, bool t2);
void wHong(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, bool t1, bool t2,
           int warpSize);
void wSlota(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, bool t1, bool t2,
            int warpSize);
// Not provided (throws "detectSCC (-a d) is not provided by this engine");
// present so that the reference's scc.cu links unchanged.
void detectSCC(uint32_t CSize, uint32_t RSize, uint32_t *Fc, uint32_t *Fr, uint32_t *Bc, uint32_t *Br, uint32_t *Pr,
               bool t1, bool t2);
void loadFullGraph(const char *filename, uint32_t *oCSize, uint32_t *oRSize, uint32_t **oFc, uint32_t **oFr,
                   uint32_t **oBc, uint32_t **oBr, uint32_t **oPr);

#endif
