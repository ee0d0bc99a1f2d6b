/*
 * Reference-arm helper -- test infrastructure only, never on the engine's path.
 *
 * Drives the reference's own populate_ion_rate_matrix (source/matrix_ion.c:444-659),
 * compiled unmodified from the reference tree by oracle/Makefile (target
 * refion) into oracle/_ref/libref_ionmat.so.  The routine reads the atomic
 * tables and the per-cell coefficient arrays from globals declared in
 * source/atomic.h; this file defines those globals, fills them from plain
 * arrays and returns the assembled nions x nions matrix and right-hand side.
 * The link keeps only what populate_ion_rate_matrix needs (section garbage
 * collection, one exported symbol), so none of the physics around it is built.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include "atomic.h"
#include "python.h"

int nelements, nions, n_inner_tot, n_charge_exchange;
ElemPtr ele;
IonPtr ion;
Topbase_phot inner_cross[N_INNER * NIONS];
Inner_elec_yield inner_elec_yield[N_INNER * NIONS];
double dr_coeffs[NIONS], di_coeffs[NIONS], qrecomb_coeffs[NIONS];
Charge_exchange charge_exchange[MAX_CHARGE_EXCHANGE];
double charge_exchange_recomb_rates[NIONS], charge_exchange_ioniz_rates[MAX_CHARGE_EXCHANGE];

/* Element e: atomic number elem_z[e], ions elem_first[e] .. with highest stage
 * elem_istate_max[e].  Ion i: element index ion_nelem[i], stage ion_istate[i]
 * (1 = neutral), flags ion_di[i] (dere_di_flag) and ion_dr[i] (drflag).
 * Inner-shell rate m depopulates ion inner_nion[m] with electron-yield row
 * inner_yield[m] (-1: no yield data) of yield_prob (n_yield x 10).  Charge
 * exchange entry m ionises ion cx_nion1[m] against ion cx_nion2[m].
 * Coefficients: pi, rr, di, qr, dr, cxr per ion; cxi per charge-exchange
 * entry; inner per inner-shell rate.  Output: A (nions x nions, row-major), b.
 * Returns populate_ion_rate_matrix's value, or -1 for sizes outside the
 * reference's static tables. */
int refion_assemble(int n_ions, int n_elem, const int *elem_z, const int *elem_first, const int *elem_istate_max,
                    const int *ion_nelem, const int *ion_istate, const int *ion_di, const int *ion_dr, int n_inner,
                    const int *inner_nion, const int *inner_yield, int n_yield, const double *yield_prob, int ncx,
                    const int *cx_nion1, const int *cx_nion2, const double *pi, const double *rr, const double *di,
                    const double *qr, const double *dr, const double *cxr, const double *cxi, const double *inner,
                    double xne, double nh1, double nh2, double *A, double *b)
{
  if (n_ions < 1 || n_ions > NIONS || n_elem < 1 || n_inner < 0 || n_inner > N_INNER * NIONS || n_yield < 0 ||
      n_yield > N_INNER * NIONS || ncx < 0 || ncx > MAX_CHARGE_EXCHANGE)
    return -1;
  nions = n_ions;
  nelements = n_elem;
  n_inner_tot = n_inner;
  n_charge_exchange = ncx;
  ele = calloc((size_t) n_elem, sizeof (*ele));
  ion = calloc((size_t) n_ions, sizeof (*ion));
  double *rm = malloc(sizeof (double) * (size_t) n_ions * (size_t) n_ions);
  if (!ele || !ion || !rm)
  {
    free(ele);
    free(ion);
    free(rm);
    return -1;
  }
  for (int e = 0; e < n_elem; e++)
  {
    ele[e].z = elem_z[e];
    ele[e].firstion = elem_first[e];
    ele[e].istate_max = elem_istate_max[e];
  }
  for (int i = 0; i < n_ions; i++)
  {
    ion[i].nelem = ion_nelem[i];
    ion[i].z = elem_z[ion_nelem[i]];
    ion[i].istate = ion_istate[i];
    ion[i].dere_di_flag = ion_di[i];
    ion[i].drflag = ion_dr[i];
    di_coeffs[i] = di[i];
    qrecomb_coeffs[i] = qr[i];
    dr_coeffs[i] = dr[i];
    charge_exchange_recomb_rates[i] = cxr[i];
  }
  for (int m = 0; m < n_inner; m++)
  {
    memset(&inner_cross[m], 0, sizeof (inner_cross[m]));
    inner_cross[m].nion = inner_nion[m];
    inner_cross[m].z = ion[inner_nion[m]].z;
    inner_cross[m].istate = ion[inner_nion[m]].istate;
    inner_cross[m].n_elec_yield = inner_yield[m];
  }
  for (int y = 0; y < n_yield; y++)
    for (int k = 0; k < 10; k++)
      inner_elec_yield[y].prob[k] = yield_prob[y * 10 + k];
  for (int m = 0; m < ncx; m++)
  {
    memset(&charge_exchange[m], 0, sizeof (charge_exchange[m]));
    charge_exchange[m].nion1 = cx_nion1[m];
    charge_exchange[m].nion2 = cx_nion2[m];
    charge_exchange_ioniz_rates[m] = cxi[m];
  }
  /* populate_ion_rate_matrix takes its rate arrays as non-const */
  double *pi_w = malloc(sizeof (double) * (size_t) n_ions), *rr_w = malloc(sizeof (double) * (size_t) n_ions);
  double *in_w = malloc(sizeof (double) * (size_t) (n_inner > 0 ? n_inner : 1));
  if (!pi_w || !rr_w || !in_w)
  {
    free(pi_w);
    free(rr_w);
    free(in_w);
    free(rm);
    free(ele);
    free(ion);
    return -1;
  }
  memcpy(pi_w, pi, sizeof (double) * (size_t) n_ions);
  memcpy(rr_w, rr, sizeof (double) * (size_t) n_ions);
  if (n_inner > 0)
    memcpy(in_w, inner, sizeof (double) * (size_t) n_inner);
  int rc = populate_ion_rate_matrix((double (*)[n_ions]) rm, pi_w, in_w, rr_w, b, xne, nh1, nh2);
  memcpy(A, rm, sizeof (double) * (size_t) n_ions * (size_t) n_ions);
  free(pi_w);
  free(rr_w);
  free(in_w);
  free(rm);
  free(ele);
  free(ion);
  ele = NULL;
  ion = NULL;
  return rc;
}
