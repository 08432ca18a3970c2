/* Link test of the drop-in (test infrastructure): a caller with lioamber's
 * link line, this library first and the reference's g2g (XC and the analytic
 * integrals) after it, binding the entry points the way lioamber's Fortran
 * does (lioamber/init_lio.f90:139-142,181, lioamber/drive.f90:176-180,
 * lioamber/SCF.f90:296-299).
 *
 * Checks: g2g_* resolve to libg2g_b200, aint_* to the reference's library;
 * g2g_parameter_init_ reaches the reference's too (its analytic integrals read
 * the state it records: here, the atom count); aint_query_gpu_level_ runs.
 * Exit status 0 when all hold. No GPU is needed. */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stdbool.h>
#include <stdio.h>
#include <string.h>

#include "g2g.h"

void aint_query_gpu_level_(int* gpu_level_out);
int ref_bound_atoms(void);

static double r[3] = {0.1, 0.2, 0.3};
static double Rm[55], e1[50 * 3], e2[116 * 3], e3[194 * 3], w1[50], w2[116], w3[194];
static unsigned Iz[1] = {1}, Nr[55], Nr2[55], Nuc[1] = {1}, ncont[1] = {1}, nshell[3] = {1, 0, 0};
static double c[13] = {1.0}, a[13] = {1.0}, rho[1] = {1.0}, fock[1], fockb[1], rhoa[1], rhob[1];

static const char* lib_of(void* sym) {
  Dl_info info;
  return dladdr(sym, &info) && info.dli_fname ? info.dli_fname : "?";
}

int main(void) {
  for (int i = 0; i < 55; i++) {
    Rm[i] = 0.5;
    Nr[i] = Nr2[i] = 10;
  }
  double fgm = 0.0, lcs = 8.0, sr = 0.6;
  bool aaf = false, eai = true, rzw = true, open = false, libxc = false;
  unsigned mppc = 1, mfe = 10, timer = 0, verbose = 0;
  unsigned norm = 1, natom = 1, max_atoms = 1, ngauss = 1, M = 1, nco = 1, nunp = 0, nopt = 0, iexch = 9, ex = 0,
           ec = 0;
  g2g_init_();
  g2g_set_options_(&fgm, &lcs, &sr, &aaf, &eai, &rzw, &mppc, &mfe, &timer, &verbose);
  g2g_parameter_init_(&norm, &natom, &max_atoms, &ngauss, r, Rm, Iz, Nr, Nr2, Nuc, &M, ncont, nshell, c, a, rho, fock,
                      fockb, rhoa, rhob, &nco, &open, &nunp, &nopt, &iexch, e1, e2, e3, w1, w2, w3, &libxc, &ex, &ec);
  int level = -1;
  aint_query_gpu_level_(&level);
  const char* g2g_lib = lib_of((void*)g2g_solve_groups_);
  const char* init_lib = lib_of((void*)g2g_parameter_init_);
  const char* aint_lib = lib_of((void*)aint_query_gpu_level_);
  const int atoms = ref_bound_atoms();
  printf("g2g_solve_groups_ %s\ng2g_parameter_init_ %s\naint_query_gpu_level_ %s (level %d)\n"
         "atoms recorded by the reference's g2g_parameter_init_: %d\n",
         g2g_lib, init_lib, aint_lib, level, atoms);
  const int ok = strstr(g2g_lib, "libg2g_b200") && strstr(init_lib, "libg2g_b200") && strstr(aint_lib, "lio_g2g") &&
                 level == 0 && atoms == 1;
  return ok ? 0 : 1;
}
