/*
 * Reference-arm helper -- test infrastructure only, never on the engine's path.
 *
 * Drives the reference's own calc_matom_matrix (source/macro_accelerate.c:31-348),
 * compiled unmodified from the reference tree by oracle/Makefile (target
 * refmatom) into oracle/_ref/libref_matom.so together with the reference's
 * matrix_cpu.c and GSL for its inversion.  The routine reads the macro-atom
 * tables (xconfig[], line[], phot_top[], auger_macro[], macromain[]) from
 * globals and the per-cell physics through a21, p_escape, q21, b12, q12,
 * q_recomb, q_ioniz and den_config.  This file defines those globals and
 * functions: the functions return per-line, per-continuum and per-level
 * values the caller supplies, and the cell's k-packet cooling rates are
 * marked known, so the routine's own fill_kpkt_rates keeps them.  The result
 * is the routine's B = N^-1 diag(R).
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "atomic.h"
#include "python.h"

int nlevels_macro, nlines, nphot_total;
ConfigPtr xconfig;
AugerPtr auger_macro;
LinePtr line, lin_ptr[NLINES];
Topbase_phot phot_top[NLEVELS];
MacroPtr macromain;
IonPtr ion;
struct geometry geo;
double DENSITY_PHOT_MIN;
WindPtr wmain;
struct xbands xband;

static const double *s_a21, *s_pesc, *s_q21, *s_b12, *s_q12, *s_qrec, *s_qion, *s_den;

double a21(struct lines *line_ptr) { return s_a21[line_ptr - line]; }
double p_escape(struct lines *line_ptr, PlasmaPtr xplasma) { (void) xplasma; return s_pesc[line_ptr - line]; }
double q21(struct lines *line_ptr, double t) { (void) t; return s_q21[line_ptr - line]; }
double b12(struct lines *line_ptr) { return s_b12[line_ptr - line]; }
double q12(struct lines *line_ptr, double t) { (void) t; return s_q12[line_ptr - line]; }
double q_recomb(struct topbase_phot *cont_ptr, double t) { (void) t; return s_qrec[cont_ptr - phot_top]; }
double q_ioniz(struct topbase_phot *cont_ptr, double t) { (void) t; return s_qion[cont_ptr - phot_top]; }
double den_config(PlasmaPtr xplasma, int nconf) { (void) xplasma; return s_den[nconf]; }
/* fill_kpkt_rates (macro_accelerate.c) keeps the stored k-packet cooling rates
   when kpkt_rates_known is set, as here; these three are then never called */
double two_level_atom(struct lines *l, PlasmaPtr x, double *d1, double *d2) { (void) l; (void) x; *d1 = *d2 = 0.0; return 0.0; }
double alpha_sp(struct topbase_phot *c, PlasmaPtr x, int i) { (void) c; (void) x; (void) i; return 0.0; }
double total_free(PlasmaPtr x, double t, double f1, double f2) { (void) x; (void) t; (void) f1; (void) f2; return 0.0; }
int init_dummy_phot(PhotPtr p) { (void) p; return 0; }
int sane_check(double x) { return isfinite(x) ? 0 : -1; }

/* Level u has n_bbd[u] downward bound-bound jumps (line indices bbd_line[...],
 * levels in order), n_bbu[u] upward ones, n_bfd[u] / n_bfu[u] bound-free
 * jumps (continuum indices), and Auger entry aug_idx[u] (-1: none) with
 * n_aug[u] channels; Auger entry k has targets aug_target[4k..] and
 * branching ratios aug_branch[4k..] and total rate aug_A[k].  Line i runs from
 * level line_lo[i] to line_up[i]; continuum i from phot_lo[i] to phot_up[i];
 * the macro_info flags mark macro-atom lines / continua.  Per-cell values:
 * a21, p_escape, q21, b12, q12 per line; q_recomb, q_ioniz per continuum;
 * jbar / gamma / alpha_st / recomb_sp per jump estimator (upward bound-bound,
 * upward bound-free twice, downward bound-free, levels in order); den per
 * level; the k-packet cooling rates.  Returns 0, or -1 for sizes outside the
 * reference's static tables; B receives (nlev + 1)^2 values, row-major. */
int refmatom_b(int nlev, const double *ex, const int *n_bbd, const int *bbd_line, const int *n_bbu,
               const int *bbu_line, const int *n_bfd, const int *bfd_phot, const int *n_bfu, const int *bfu_phot,
               const int *aug_idx, const int *n_aug, int naug, const int *aug_target, const double *aug_A,
               const double *aug_branch, int nline, const int *line_lo, const int *line_up, const int *line_macro,
               int nphot, const int *phot_lo, const int *phot_up, const int *phot_macro, const double *a21v,
               const double *pesc, const double *q21v, const double *b12v, const double *q12v, const double *qrec,
               const double *qion, const double *jbar, const double *gamma, const double *alpha_st,
               const double *recomb_sp, const double *den, const double *cool_bb, const double *cool_bf,
               double cool_bftot, double cool_adiabatic, double cool_ff, double cool_ff_lofreq, double t_e, double ne,
               double density_phot_min, double *B)
{
  if (nlev < 1 || nline < 0 || nline > NLINES || nphot < 0 || nphot > NLEVELS || naug < 0)
    return -1;
  int nbbu_tot = 0, nbfu_tot = 0, nbfd_tot = 0;
  for (int u = 0; u < nlev; u++)
  {
    if (n_bbd[u] > NBBJUMPS || n_bbu[u] > NBBJUMPS || n_bfd[u] > NBFJUMPS || n_bfu[u] > NBFJUMPS ||
        n_aug[u] > NAUGER_ELECTRONS)
      return -1;
    nbbu_tot += n_bbu[u];
    nbfu_tot += n_bfu[u];
    nbfd_tot += n_bfd[u];
  }
  nlevels_macro = nlev;
  nlines = nline;
  nphot_total = nphot;
  DENSITY_PHOT_MIN = density_phot_min;
  memset(&geo, 0, sizeof (geo));
  geo.macro_simple = 0;
  xconfig = calloc((size_t) nlev, sizeof (*xconfig));
  line = calloc((size_t) (nline > 0 ? nline : 1), sizeof (*line));
  auger_macro = calloc((size_t) (naug > 0 ? naug : 1), sizeof (*auger_macro));
  macromain = calloc(1, sizeof (*macromain));
  ion = calloc(1, sizeof (*ion));
  PlasmaPtr xp = calloc(1, sizeof (*xp));
  double **mm = calloc((size_t) nlev + 1, sizeof (double *));
  double *store = calloc((size_t) (nlev + 1) * (size_t) (nlev + 1), sizeof (double));
  if (!xconfig || !line || !auger_macro || !macromain || !ion || !xp || !mm || !store)
    return -1;
  for (int r = 0; r <= nlev; r++)
    mm[r] = store + (size_t) r * (size_t) (nlev + 1);
  int ib = 0, ibu = 0, ifd = 0, ifu = 0;
  for (int u = 0; u < nlev; u++)
  {
    xconfig[u].ex = ex[u];
    xconfig[u].nion = 0;
    xconfig[u].n_bbd_jump = n_bbd[u];
    for (int n = 0; n < n_bbd[u]; n++)
      xconfig[u].bbd_jump[n] = bbd_line[ib++];
    xconfig[u].n_bbu_jump = n_bbu[u];
    xconfig[u].bbu_indx_first = ibu;
    for (int n = 0; n < n_bbu[u]; n++)
      xconfig[u].bbu_jump[n] = bbu_line[ibu++];
    xconfig[u].n_bfd_jump = n_bfd[u];
    xconfig[u].bfd_indx_first = ifd;
    for (int n = 0; n < n_bfd[u]; n++)
      xconfig[u].bfd_jump[n] = bfd_phot[ifd++];
    xconfig[u].n_bfu_jump = n_bfu[u];
    xconfig[u].bfu_indx_first = ifu;
    for (int n = 0; n < n_bfu[u]; n++)
      xconfig[u].bfu_jump[n] = bfu_phot[ifu++];
    xconfig[u].iauger = aug_idx[u];
    xconfig[u].nauger = n_aug[u];
  }
  for (int k = 0; k < naug; k++)
  {
    auger_macro[k].Avalue_auger = aug_A[k];
    for (int n = 0; n < NAUGER_ELECTRONS; n++)
    {
      auger_macro[k].nconfig_target[n] = aug_target[k * NAUGER_ELECTRONS + n];
      auger_macro[k].branching_ratio[n] = aug_branch[k * NAUGER_ELECTRONS + n];
    }
  }
  for (int i = 0; i < nline; i++)
  {
    line[i].nconfigl = line_lo[i];
    line[i].nconfigu = line_up[i];
    line[i].macro_info = line_macro[i];
  }
  for (int i = 0; i < nphot; i++)
  {
    memset(&phot_top[i], 0, sizeof (phot_top[i]));
    phot_top[i].nlev = phot_lo[i];
    phot_top[i].uplev = phot_up[i];
    phot_top[i].macro_info = phot_macro[i];
  }
  s_a21 = a21v;
  s_pesc = pesc;
  s_q21 = q21v;
  s_b12 = b12v;
  s_q12 = q12v;
  s_qrec = qrec;
  s_qion = qion;
  s_den = den;
  /* the routine reads these arrays only */
  macromain[0].jbar_old = (double *) jbar;
  macromain[0].gamma_old = (double *) gamma;
  macromain[0].alpha_st_old = (double *) alpha_st;
  macromain[0].recomb_sp = (double *) recomb_sp;
  macromain[0].cooling_bb = (double *) cool_bb;
  macromain[0].cooling_bf_col = (double *) cool_bf;
  macromain[0].cooling_bftot = cool_bftot;
  macromain[0].cooling_adiabatic = cool_adiabatic;
  macromain[0].cooling_ff = cool_ff;
  macromain[0].cooling_ff_lofreq = cool_ff_lofreq;
  macromain[0].kpkt_rates_known = TRUE;
  xp->nplasma = 0;
  xp->t_e = t_e;
  xp->ne = ne;
  calc_matom_matrix(xp, mm);
  memcpy(B, store, sizeof (double) * (size_t) (nlev + 1) * (size_t) (nlev + 1));
  free(store);
  free(mm);
  free(xp);
  free(ion);
  free(macromain);
  free(auger_macro);
  free(line);
  free(xconfig);
  line = NULL;
  xconfig = NULL;
  return 0;
}
