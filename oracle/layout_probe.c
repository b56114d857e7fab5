/*
 * Struct-layout probe (test infrastructure).  Compiled once against the
 * reference's headers (-DPROBE_REFERENCE_HEADERS; include/iga.h, nurbs.h,
 * bc.h, phys.h, snes.h, iocomm.h of IGAP4STANDARD) and once against
 * include/igap4_structs.h; the tests compare the two tables to show the
 * drop-in library receives byte-identical structs.
 */
#include <stddef.h>
#ifdef PROBE_REFERENCE_HEADERS
#include "snesiga.h"
#include "iocomm.h"
#define PROBE_FN layout_probe_reference
#else
#include "igap4_structs.h"
#define PROBE_FN layout_probe_ours
#endif

#define S(T) out[n++] = (long)sizeof(T)
#define O(T, m) out[n++] = (long)offsetof(T, m)

int PROBE_FN(long *out)
{
    int n = 0;
    S(Phys); O(Phys, ndim); O(Phys, ndof); O(Phys, torder); O(Phys, sorder); O(Phys, par_mat);
    O(Phys, ndensity); O(Phys, nfield); O(Phys, residual); O(Phys, tangent); O(Phys, field);
    O(Phys, density); O(Phys, densityb); O(Phys, assert_par_mat);
    S(Nurbs); O(Nurbs, porder); O(Nurbs, nelem); O(Nurbs, nbasis); O(Nurbs, nknot); O(Nurbs, knotVector);
    O(Nurbs, nboun); O(Nurbs, boun); O(Nurbs, nsendPart); O(Nurbs, sendPart); O(Nurbs, nrecvPart);
    O(Nurbs, recvPart); O(Nurbs, sendBlock); O(Nurbs, recvBlock); O(Nurbs, universalIdx_temp);
    O(Nurbs, bc_periodic); O(Nurbs, nelem_global); O(Nurbs, knotVector_global);
    S(BC); O(BC, bc_type); O(BC, par_periodic); O(BC, par_dirichlet); O(BC, par_neumann);
    S(IGA); O(IGA, phys); O(IGA, nurbs); O(IGA, bc); O(IGA, U_hist); O(IGA, nselfIdx); O(IGA, selfIdx);
    O(IGA, nsendIdx); O(IGA, sendIdx); O(IGA, sendPtr); O(IGA, nrecvIdx); O(IGA, recvIdx);
    O(IGA, recvPtr); O(IGA, globalIdx);
    S(SNESAssmbl); O(SNESAssmbl, snes_Residual); O(SNESAssmbl, snes_Tangent); O(SNESAssmbl, Residual_);
    O(SNESAssmbl, Tangent_); O(SNESAssmbl, snes); O(SNESAssmbl, U); O(SNESAssmbl, converged);
    S(IOcomm); O(IOcomm, nDof); O(IOcomm, nDof_array); O(IOcomm, iDof_displ_array);
    O(IOcomm, nDof_global); O(IOcomm, universalIdx);
    return n;
}
