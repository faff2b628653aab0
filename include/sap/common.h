/* The enumerations of the reference's sap/common.h:67-98 (same names and
 * values), for code written against sap::Options, plus the FGMRES solver
 * extension of libsap_b200. */
#ifndef SAP_B200_FACADE_COMMON_H
#define SAP_B200_FACADE_COMMON_H

#include "../sap_b200.h"

namespace sap {

enum KrylovSolverType {
  BiCGStab_C = SAP_BICGSTAB_C,  // CUSP solvers: not provided (setup/solve report SAP_ERR_UNSUPPORTED)
  GMRES_C = SAP_GMRES_C,
  CG_C = SAP_CG_C,
  CR_C = SAP_CR_C,
  BiCGStab1 = SAP_BICGSTAB1,
  BiCGStab2 = SAP_BICGSTAB2,
  BiCGStab = SAP_BICGSTAB,
  MINRES = SAP_MINRES,
  FGMRES = SAP_FGMRES  // extension: flexible GMRES(50) with FP64 Arnoldi
};

enum FactorizationMethod { LU_UL = SAP_LU_UL, LU_only = SAP_LU_ONLY };

enum PreconditionerType { Spike = SAP_PRECOND_SPIKE, Block = SAP_PRECOND_BLOCK, None = SAP_PRECOND_NONE };

}  // namespace sap

#endif
