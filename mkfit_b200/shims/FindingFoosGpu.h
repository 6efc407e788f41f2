// FindingFoosGpu: the reference's finding operator table (FindingFoos,
// mkFit/FindingFoos.h:10-38) with its chi2 and update operators on the GPU,
// for MkFinder call sites: the functions below have the reference's
// COMPUTE_CHI2_ARGS / UPDATE_PARAM_ARGS signatures and run
// mkfg_op_propagate_chi2 / mkfg_op_propagate_update on the Matriplex
// storage as it is (element stride NN). The table's third member is a
// pointer to an MkBase member function, which only MkBase can provide: the
// tables returned here keep the reference's own PropagateTracksToR / ToZ
// there, and propagate_to_r / propagate_to_z below are the GPU forms of
// those two for an MkBase object.
//
// Header only; compile against the reference's headers and link
// libmkfit_b200.so. set_context() names the library context the operators
// use (one per thread, as the reference's worker pools); errors throw
// std::runtime_error with the library's message.
#ifndef MKFIT_B200_SHIMS_FINDINGFOOSGPU_H
#define MKFIT_B200_SHIMS_FINDINGFOOSGPU_H

#include <stdexcept>
#include <string>

#include "mkFit/FindingFoos.h"
#include "mkFit/MkBase.h"
#include "mkfit_b200.h"

namespace mkfit {

class FindingFoosGpu {
 public:
  static void set_context(mkfg_context* ctx) { ctx_() = ctx; }

  // kalmanPropagateAndComputeChi2 / ...Endcap.
  static void compute_chi2_barrel(const MPlexLS& psErr, const MPlexLV& psPar, const MPlexQI& inChg,
                                  const MPlexHS& msErr, const MPlexHV& msPar, MPlexQF& outChi2,
                                  MPlexLV& propPar, const int N_proc, const PropagationFlags pf) {
    chi2(0, psErr, psPar, inChg, msErr, msPar, outChi2, propPar, N_proc, pf);
  }
  static void compute_chi2_endcap(const MPlexLS& psErr, const MPlexLV& psPar, const MPlexQI& inChg,
                                  const MPlexHS& msErr, const MPlexHV& msPar, MPlexQF& outChi2,
                                  MPlexLV& propPar, const int N_proc, const PropagationFlags pf) {
    chi2(1, psErr, psPar, inChg, msErr, msPar, outChi2, propPar, N_proc, pf);
  }
  // kalmanPropagateAndUpdate / ...Endcap.
  static void update_barrel(const MPlexLS& psErr, const MPlexLV& psPar, MPlexQI& Chg,
                            const MPlexHS& msErr, const MPlexHV& msPar, MPlexLS& outErr,
                            MPlexLV& outPar, const int N_proc, const PropagationFlags pf) {
    update(0, psErr, psPar, Chg, msErr, msPar, outErr, outPar, N_proc, pf);
  }
  static void update_endcap(const MPlexLS& psErr, const MPlexLV& psPar, MPlexQI& Chg,
                            const MPlexHS& msErr, const MPlexHV& msPar, MPlexLS& outErr,
                            MPlexLV& outPar, const int N_proc, const PropagationFlags pf) {
    update(1, psErr, psPar, Chg, msErr, msPar, outErr, outPar, N_proc, pf);
  }
  // MkBase::PropagateTracksToR / ToZ on mb: Err/Par[iC] -> Err/Par[iP].
  static void propagate_to_r(MkBase& mb, float r, const int N_proc, const PropagationFlags pf) {
    propagate(0, mb, r, N_proc, pf);
  }
  static void propagate_to_z(MkBase& mb, float z, const int N_proc, const PropagationFlags pf) {
    propagate(1, mb, z, N_proc, pf);
  }

  static const FindingFoos& get_finding_foos(bool is_barrel) {
    static const FindingFoos brl(compute_chi2_barrel, update_barrel, &MkBase::PropagateTracksToR);
    static const FindingFoos ec(compute_chi2_endcap, update_endcap, &MkBase::PropagateTracksToZ);
    return is_barrel ? brl : ec;
  }

 private:
  static mkfg_context*& ctx_() {
    static thread_local mkfg_context* c = nullptr;
    return c;
  }
  static mkfg_context* ctx() {
    if (!ctx_()) throw std::runtime_error("FindingFoosGpu: set_context was not called");
    return ctx_();
  }
  static uint32_t bits(const PropagationFlags& p) {
    return (p.use_param_b_field ? 1u : 0u) | (p.apply_material ? 2u : 0u);
  }
  static void check(int rc) {
    if (rc == MKFG_OK) return;
    char msg[512];
    mkfg_last_error(msg, sizeof(msg));
    throw std::runtime_error(std::string("mkfit_b200: ") + msg);
  }
  static void chi2(int endcap, const MPlexLS& psErr, const MPlexLV& psPar, const MPlexQI& inChg,
                   const MPlexHS& msErr, const MPlexHV& msPar, MPlexQF& outChi2,
                   MPlexLV& propPar, const int N_proc, const PropagationFlags pf) {
    propPar = psPar;  // as the reference: lanes past N_proc keep the input
    check(mkfg_op_propagate_chi2(ctx(), endcap, N_proc, NN, psPar.fArray, psErr.fArray,
                                 inChg.fArray, msPar.fArray, msErr.fArray, bits(pf),
                                 outChi2.fArray, propPar.fArray));
  }
  static void update(int endcap, const MPlexLS& psErr, const MPlexLV& psPar, MPlexQI& Chg,
                     const MPlexHS& msErr, const MPlexHV& msPar, MPlexLS& outErr, MPlexLV& outPar,
                     const int N_proc, const PropagationFlags pf) {
    check(mkfg_op_propagate_update(ctx(), endcap, N_proc, NN, psPar.fArray, psErr.fArray,
                                   Chg.fArray, msPar.fArray, msErr.fArray, bits(pf),
                                   outPar.fArray, outErr.fArray, Chg.fArray));
  }
  static void propagate(int endcap, MkBase& mb, float target, const int N_proc,
                        const PropagationFlags pf) {
    float t[NN];
    for (int n = 0; n < NN; ++n) t[n] = target;
    check(mkfg_op_propagate(ctx(), endcap, N_proc, NN, mb.Par[MkBase::iC].fArray,
                            mb.Err[MkBase::iC].fArray, mb.Chg.fArray, t, bits(pf),
                            mb.Par[MkBase::iP].fArray, mb.Err[MkBase::iP].fArray));
  }
};

}  // namespace mkfit

#endif
