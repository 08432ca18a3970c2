/* Test infrastructure only: the oracle (see g2g_oracle.h). Plain C, FP64,
 * compiled with -ffp-contract=off and no -march (no fused multiply-add), so
 * the grid partition reproduces the reference bit for bit. Each function cites
 * the reference lines it restates. */
#include "g2g_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXC 13
#define FL(x) ((double)(float)(x))

/* ------------------------------------------------------------------ containers */
typedef struct {
  int atom, shell, point;
  double x, y, z, w;
} pt_t;

typedef struct {
  pt_t* v;
  int n, cap;
} ptvec;

static void pv_push(ptvec* a, pt_t p) {
  if (a->n == a->cap) {
    a->cap = a->cap ? 2 * a->cap : 64;
    a->v = (pt_t*)realloc(a->v, (size_t)a->cap * sizeof(pt_t));
  }
  a->v[a->n++] = p;
}

typedef struct {
  ptvec p;
  int* funcs; /* simple functions, global index of first component */
  int nf;
  int* nucs;
  int nn;
  int s, pc, dc;
  int sphere;
  long long cost;
} group_t;

static int total_functions(const group_t* g) { return g->s + 3 * g->pc + 6 * g->dc; }

/* ------------------------------------------------------------ partition */
/* g2g/partition.cpp:230-254 */
static int significant(int type, double exponent, double d2, unsigned mfe) {
  if (type == 1) return (exponent * d2 < mfe - log(pow((2. * exponent / M_PI), 3)) / 4);
  double x = 1, delta;
  double factor = pow((2.0 * exponent / M_PI), 3);
  factor = sqrt(factor * 4.0 * exponent);
  double norm = (type == 3 ? sqrt(factor) : fabs(factor));
  do {
    double div = (type == 3 ? log(x) : 2 * log(x));
    double x1 = sqrt((mfe - log(norm) + div) / exponent);
    delta = fabs(x - x1);
    x = x1;
  } while (delta > 0.1);
  return (sqrt(d2) < x);
}

/* g2g/classify_functions.cpp:13-65 */
static void classify(const oracle_system* s, const double* dists, const double* min_exp, group_t* g) {
  char* seen = (char*)calloc((size_t)s->natoms, 1);
  int cap = s->s_funcs + s->p_funcs + s->d_funcs + 1;
  g->funcs = (int*)malloc(sizeof(int) * (size_t)cap);
  g->nf = g->s = g->pc = g->dc = 0;
  int f = 0;
  const int se = s->s_funcs, pe = se + 3 * s->p_funcs, de = pe + 6 * s->d_funcs;
  for (; f < se; f++)
    if (s->assign_all_functions || significant(1, min_exp[f], dists[s->nuc[f]], s->max_function_exponent)) {
      g->funcs[g->nf++] = f;
      g->s++;
      seen[s->nuc[f]] = 1;
    }
  for (; f < pe; f += 3)
    if (s->assign_all_functions || significant(3, min_exp[f], dists[s->nuc[f]], s->max_function_exponent)) {
      g->funcs[g->nf++] = f;
      g->pc++;
      seen[s->nuc[f]] = 1;
    }
  for (; f < de; f += 6)
    if (s->assign_all_functions || significant(6, min_exp[f], dists[s->nuc[f]], s->max_function_exponent)) {
      g->funcs[g->nf++] = f;
      g->dc++;
      seen[s->nuc[f]] = 1;
    }
  g->nucs = (int*)malloc(sizeof(int) * (size_t)(s->natoms + 1));
  g->nn = 0;
  for (int a = 0; a < s->natoms; a++)
    if (seen[a]) g->nucs[g->nn++] = a;
  free(seen);
}

static double dist3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

/* g2g/cpu/weight.cpp:13-112 (Becke with atomic-size adjustment, 3 smoothing steps) */
static double becke_u(double u, double rj, double rk) {
  double x = rj / rk;
  x = (x - 1.0) / (x + 1.0);
  u += (x / (x * x - 1.0)) * (1.0 - u * u);
  u = 1.5 * u - 0.5 * (u * u * u);
  u = 1.5 * u - 0.5 * (u * u * u);
  u = 1.5 * u - 0.5 * (u * u * u);
  return 0.5 * (1.0 - u);
}

static void weights(const oracle_system* s, const double* rm, const double* adist, group_t* g) {
  const int nn = g->nn;
  for (int q = 0; q < g->p.n; q++) {
    pt_t* pt = &g->p.v[q];
    double Pt = 0.0, Pa = 0.0;
    int own = 0;
    for (int j = 0; j < nn; j++) {
      const int aj = g->nucs[j];
      double Pc = 1.0;
      for (int k = 0; k < nn; k++) {
        const int ak = g->nucs[k];
        if (ak == aj) continue;
        double u = (dist3(pt->x - s->x[aj], pt->y - s->y[aj], pt->z - s->z[aj]) -
                    dist3(pt->x - s->x[ak], pt->y - s->y[ak], pt->z - s->z[ak])) /
                   adist[(size_t)aj * s->natoms + ak];
        Pc *= becke_u(u, rm[aj], rm[ak]);
        if (Pc == 0.0) break;
      }
      if (aj == pt->atom) {
        own = 1;
        Pa = Pc;
        if (Pa == 0.0) break;
      }
      Pt += Pc;
    }
    if (!own) {
      const int aj = pt->atom;
      Pa = 1.0;
      for (int k = 0; k < nn; k++) {
        const int ak = g->nucs[k];
        double u = (dist3(pt->x - s->x[aj], pt->y - s->y[aj], pt->z - s->z[aj]) -
                    dist3(pt->x - s->x[ak], pt->y - s->y[ak], pt->z - s->z[ak])) /
                   adist[(size_t)aj * s->natoms + ak];
        Pa *= becke_u(u, rm[aj], rm[ak]);
        if (Pa == 0.0) break;
      }
    }
    pt->w *= (Pt == 0.0 ? 0.0 : (Pa / Pt));
  }
  if (s->remove_zero_weights) {
    int k = 0;
    for (int q = 0; q < g->p.n; q++)
      if (g->p.v[q].w != 0.0) g->p.v[k++] = g->p.v[q];
    g->p.n = k;
  }
}

static int cmp_cost(const void* a, const void* b) {
  const group_t* x = (const group_t*)a;
  const group_t* y = (const group_t*)b;
  return (x->cost > y->cost) - (x->cost < y->cost);
}

/* g2g/regenerate_partition.cpp:161-466. Returns groups (cubes, then spheres). */
static group_t* build_groups(const oracle_system* s, int* ngroups_out) {
  const int na = s->natoms;
  double* rm = (double*)malloc(sizeof(double) * (size_t)na);
  unsigned* nsh = (unsigned*)malloc(sizeof(unsigned) * (size_t)na);
  for (int a = 0; a < na; a++) {
    rm[a] = s->rm_by_Z[s->Z[a]];
    nsh[a] = s->shells_by_Z[s->Z[a]];
  }
  double* adist = (double*)malloc(sizeof(double) * (size_t)na * na);
  for (int i = 0; i < na; i++)
    for (int j = 0; j < na; j++)
      adist[(size_t)i * na + j] = dist3(s->x[i] - s->x[j], s->y[i] - s->y[j], s->z[i] - s->z[j]);
  double min_type[120];
  for (int t = 0; t < 120; t++) min_type[t] = DBL_MAX;
  double* min_exp = (double*)malloc(sizeof(double) * (size_t)s->M);
  for (int i = 0; i < s->M; i++) {
    min_exp[i] = DBL_MAX;
    const int t = s->Z[s->nuc[i]] - 1;
    for (int k = 0; k < s->ncont[i]; k++) {
      const double a = s->a[i * MAXC + k];
      if (a < min_type[t]) min_type[t] = a;
      if (a < min_exp[i]) min_exp[i] = a;
    }
  }
  double x0[3] = {0, 0, 0}, x1[3] = {0, 0, 0};
  for (int a = 0; a < na; a++) {
    const double pos[3] = {s->x[a], s->y[a], s->z[a]};
    const double r = 2 * sqrt(s->max_function_exponent / min_type[s->Z[a] - 1]);
    for (int d = 0; d < 3; d++) {
      if (a == 0) {
        x0[d] = pos[d] - r;
        x1[d] = pos[d] + r;
      } else {
        if (pos[d] - r < x0[d]) x0[d] = pos[d] - r;
        if (pos[d] + r > x1[d]) x1[d] = pos[d] + r;
      }
    }
  }
  const double lcs = s->little_cube_size;
  unsigned ps[3];
  for (int d = 0; d < 3; d++) ps[d] = (unsigned)ceil((x1[d] - x0[d]) / lcs);
  double* srad = (double*)calloc((size_t)na, sizeof(double));
  for (int a = 0; a < na; a++) {
    const unsigned inc = (unsigned)ceil(s->sphere_radius * nsh[a]);
    if (s->sphere_radius > 0 && inc > 0) {
      const double x = cos((M_PI / (nsh[a] + 1)) * (nsh[a] - inc + 1));
      srad[a] = rm[a] * (1.0 + x) / (1.0 - x);
    }
  }
  const size_t ncub = (size_t)ps[0] * ps[1] * ps[2];
  ptvec* cube = (ptvec*)calloc(ncub, sizeof(ptvec));
  ptvec* sph = (ptvec*)calloc((size_t)na, sizeof(ptvec));
  for (int a = 0; a < na; a++) {
    const unsigned ns = nsh[a];
    const double t0 = M_PI / (ns + 1);
    const unsigned inc = (unsigned)ceil(s->sphere_radius * ns);
    for (unsigned sh = 0; sh < ns; sh++) {
      const double t1 = t0 * (sh + 1);
      const double x = cos(t1);
      const double w = t0 * fabs(sin(t1));
      const double r1 = rm[a] * (1.0 + x) / (1.0 - x);
      const double wrad = w * (r1 * r1) * rm[a] * 2.0 / ((1.0 - x) * (1.0 - x));
      for (int p = 0; p < s->nang; p++) {
        pt_t q = {a, (int)sh, p, s->x[a] + s->ex[p] * r1, s->y[a] + s->ey[p] * r1, s->z[a] + s->ez[p] * r1,
                  wrad * s->ew[p]};
        if (!((x0[0] <= q.x && q.x <= x1[0]) && (x0[1] <= q.y && q.y <= x1[1]) && (x0[2] <= q.z && q.z <= x1[2])))
          continue;
        if (s->sphere_radius > 0 && sh >= (ns - inc)) {
          pv_push(&sph[a], q);
        } else {
          const unsigned cx = (unsigned)floor((q.x - x0[0]) / lcs), cy = (unsigned)floor((q.y - x0[1]) / lcs),
                         cz = (unsigned)floor((q.z - x0[2]) / lcs);
          pv_push(&cube[((size_t)cx * ps[1] + cy) * ps[2] + cz], q);
        }
      }
    }
  }
  group_t* cubes = (group_t*)calloc(ncub + 1, sizeof(group_t));
  group_t* sphs = (group_t*)calloc((size_t)na + 1, sizeof(group_t));
  int nc = 0, nsph = 0;
  double* dists = (double*)malloc(sizeof(double) * (size_t)na);
  for (unsigned i = 0; i < ps[0]; i++)
    for (unsigned j = 0; j < ps[1]; j++)
      for (unsigned k = 0; k < ps[2]; k++) {
        ptvec* pv = &cube[((size_t)i * ps[1] + j) * ps[2] + k];
        const double cc[3] = {x0[0] + i * lcs, x0[1] + j * lcs, x0[2] + k * lcs};
        for (int a = 0; a < na; a++) {
          const double pos[3] = {s->x[a], s->y[a], s->z[a]};
          double dv[3];
          for (int d = 0; d < 3; d++)
            dv[d] = pos[d] < cc[d] ? cc[d] - pos[d] : (pos[d] > (cc[d] + lcs) ? pos[d] - (cc[d] + lcs) : 0);
          dists[a] = dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2];
        }
        group_t g;
        memset(&g, 0, sizeof(g));
        classify(s, dists, min_exp, &g);
        if (g.nf == 0 || (unsigned)pv->n < s->min_points_per_cube) {
          free(g.funcs);
          free(g.nucs);
          free(pv->v);
          continue;
        }
        g.p = *pv;
        weights(s, rm, adist, &g);
        if ((unsigned)g.p.n < s->min_points_per_cube) {
          free(g.funcs);
          free(g.nucs);
          free(g.p.v);
          continue;
        }
        cubes[nc++] = g;
      }
  for (int a = 0; s->sphere_radius > 0 && a < na; a++) {
    for (int o = 0; o < na; o++) {
      if (o == a) {
        dists[o] = 0;
      } else {
        const double d = dist3(s->x[o] - s->x[a], s->y[o] - s->y[a], s->z[o] - s->z[a]);
        const double dd = (srad[a] > d ? 0 : d - srad[a]);
        dists[o] = dd * dd;
      }
    }
    group_t g;
    memset(&g, 0, sizeof(g));
    classify(s, dists, min_exp, &g);
    if ((unsigned)sph[a].n < s->min_points_per_cube) {
      free(g.funcs);
      free(g.nucs);
      free(sph[a].v);
      continue;
    }
    g.p = sph[a];
    g.sphere = 1;
    weights(s, rm, adist, &g);
    if ((unsigned)g.p.n < s->min_points_per_cube) {
      free(g.funcs);
      free(g.nucs);
      free(g.p.v);
      continue;
    }
    sphs[nsph++] = g;
  }
  for (int i = 0; i < nc; i++) {
    const long long np = cubes[i].p.n, gm = total_functions(&cubes[i]);
    cubes[i].cost = 10 * ((np * gm * (1 + gm)) / 2) + s->mincost;
  }
  for (int i = 0; i < nsph; i++) {
    const long long np = sphs[i].p.n, gm = total_functions(&sphs[i]);
    sphs[i].cost = 10 * ((np * gm * (1 + gm)) / 2) + s->mincost;
  }
  qsort(cubes, (size_t)nc, sizeof(group_t), cmp_cost);
  qsort(sphs, (size_t)nsph, sizeof(group_t), cmp_cost);
  group_t* all = (group_t*)malloc(sizeof(group_t) * (size_t)(nc + nsph + 1));
  memcpy(all, cubes, sizeof(group_t) * (size_t)nc);
  memcpy(all + nc, sphs, sizeof(group_t) * (size_t)nsph);
  *ngroups_out = nc + nsph;
  free(cubes);
  free(sphs);
  free(cube);
  free(sph);
  free(dists);
  free(srad);
  free(min_exp);
  free(adist);
  free(rm);
  free(nsh);
  return all;
}

/* --------------------------------------------------------------- functionals */
/* g2g/pointxc/calc_ldaCS.h:33-102 */
static void lda(double dens, int iexch, double* ex, double* ec, double* v) {
  *ex = *ec = *v = 0.0;
  if (dens == 0) return;
  const double y = cbrt(dens);
  const double v0 = -0.984745021842697 * y;
  *ex = -0.738558766382022447 * y;
  if (iexch == 1) {
    *v = v0;
  } else if (iexch == 2) {
    const double rs = 0.620350490899400087 / y, x1 = rs / 11.4;
    double vc;
    if (x1 > 1.0) {
      *ec = -0.0333 * (0.5 * x1 - 0.33333333333333);
      vc = 0.0111 * x1 * 0.5;
    } else {
      const double t1 = (1.0 + x1 * x1 * x1), t2 = log(1.0 + 1.0 / x1), t3 = x1 * x1;
      *ec = -0.0333 * (t1 * t2 - t3 + 0.5 * x1 - 0.33333333333333);
      vc = 0.0111 * x1 * (3.0 * t3 * t2 - t1 / (x1 * (x1 + 1.0)) - 2.0 * x1 + 0.5);
    }
    *v = v0 + *ec + vc;
  } else {
    const double rs = 0.620350490899400087 / y, x1 = sqrt(rs);
    const double Xx = rs + 3.72744 * x1 + 12.9352;
    const double t1 = 2.0 * x1 + 3.72744, t2 = log(Xx), t3 = atan(6.15199066246304849 / t1);
    const double t5 = (3.72744 * x1 + 25.8704) / x1;
    *ec = (2.0 * log(x1) - t2 + 1.21178337371132 * t3 -
           -0.0311676086789438 * (2.0 * log(x1 - -0.10498) - t2 + 1.14352579286644 * t3)) *
          0.03109205;
    const double vc = *ec - 0.005182008333 * x1 *
                                (t5 / Xx - 14.90976 / (t1 * t1 + 37.8469891110325) * 1.0329232240928 -
                                 -0.0311676086789438 * (2.0 / (x1 - -0.10498) - t1 / Xx));
    *v = v0 + vc;
  }
}

/* g2g/pointxc/gcorc.h */
static void gcor(int set, double rtrs, double* gg, double* grrs) {
  double A0, A1, B1, B2, B3, B4;
  if (set == 1) {
    A0 = FL(0.0310907f); A1 = FL(0.21370f); B1 = FL(7.5957f); B2 = FL(3.5876f); B3 = FL(1.6382f); B4 = FL(0.49294f);
  } else if (set == 2) {
    A0 = FL(0.01554535f); A1 = FL(0.20548f); B1 = FL(14.1189f); B2 = FL(6.1977f); B3 = FL(3.3662f); B4 = FL(0.62517f);
  } else {
    A0 = FL(0.0168869f); A1 = FL(0.11125f); B1 = FL(10.357f); B2 = FL(3.6231f); B3 = FL(0.88026f); B4 = FL(0.49671f);
  }
  const double Q0 = -2.0 * A0 * (1.0 + A1 * rtrs * rtrs);
  const double Q1 = 2.0 * A0 * rtrs * (B1 + rtrs * (B2 + rtrs * (B3 + B4 * rtrs)));
  const double Q2 = log(1.0 + 1.0 / Q1);
  *gg = Q0 * Q2;
  const double Q3 = A0 * (B1 / rtrs + 2.0 * B2 + rtrs * (3.0 * B3 + 4.0 * B4 * rtrs));
  *grrs = -2.0 * A0 * A1 * Q2 - Q0 * Q3 / (Q1 * (1.0 + Q1));
}

#define F43 ((double)(4.0f / 3.0f))

/* g2g/pointxc/pbeCS.h:30-185 */
static void pbe_cs(double rho, double agrad, double delgrad, double rlap, double* expbe, double* vxpbe,
                   double* ecpbe, double* vcpbe) {
  const double MIN = 1e-18;
  const double UM = FL(0.2195149727645171f), UK = FL(0.804f), UL = FL(0.273028573090195f);
  const double GAMMAINV = FL(32.1639684429148f), BETA = FL(0.06672455060314922f), DELTA = FL(2.14612633996736f);
  const double rho2 = rho * rho, rho13 = cbrt(rho);
  const double fk = cbrt(FL(29.608813203268075856503472999628f)) * rho13;
  if (rho2 > MIN) {
    const double twofk = 2.0 * fk, twofk2 = twofk * twofk, twofk3 = twofk * twofk2;
    const double s = agrad / (twofk * rho), s2 = s * s, s3 = s * s2;
    const double exlda = FL(-0.738558766382022405884230032680836f) * rho13;
    const double p0 = 1.0 + UL * s2, fxpbe = 1.0 + UK - UK / p0;
    *expbe = exlda * fxpbe;
    const double v = rlap / (twofk2 * rho), u = delgrad / (twofk3 * rho2);
    const double P2 = p0 * p0, Fs = 2.0 * UM / P2, F1 = -4.0 * UL * s * Fs, Fss = F1 / p0;
    const double vx2 = F43 * fxpbe, vx3 = v * Fs, vx4 = (u - F43 * s3) * Fss;
    *vxpbe = exlda * (vx2 - vx4 - vx3);
  } else {
    *expbe = *vxpbe = 0.0;
  }
  if (rho < (MIN * 1E6)) {
    *ecpbe = *vcpbe = 0.0;
    return;
  }
  const double pirho = 4.0 * M_PI * rho, rs = cbrt(3.0 / pirho), rtrs = sqrt(rs);
  const double sk = sqrt(4.0 * fk / M_PI), twoks = 2.0 * sk, twoks2 = twoks * twoks, twoks3 = twoks2 * twoks;
  const double t = agrad / (twoks * rho), t2 = t * t;
  const double UU = delgrad / (rho2 * twoks3), VV = rlap / (rho * twoks2);
  double ec, eurs;
  gcor(1, rtrs, &ec, &eurs);
  const double vclda = ec - rs * (double)(1.0f / 3.0f) * eurs;
  const double PON = -ec * GAMMAINV, B = DELTA / (exp(PON) - 1.0), B2 = B * B, T4 = t2 * t2;
  const double Q4 = 1.0 + B * t2, Q5 = 1.0 + B * t2 + B2 * T4;
  const double H = (BETA / DELTA) * log(1.0 + DELTA * Q4 * t2 / Q5);
  *ecpbe = ec + H;
  const double T6 = T4 * t2, RSTHRD = rs / 3.0, FAC = DELTA / B + 1.0, BEC = B2 * FAC / BETA;
  const double Q8 = (Q5 + DELTA * Q4 * t2) * Q5, Q9 = 1.0 + 2.0 * B * t2;
  const double hB = -BETA * B * (T6 / Q8) * (2.0 + B * t2), hRS = -RSTHRD * hB * BEC * eurs;
  const double FACT0 = 2.0 * DELTA - 6.0 * B, FACT1 = Q5 * Q9 + Q4 * Q9 * Q9;
  const double hBT = 2.0 * BETA * T4 * ((Q4 * Q5 * FACT0 - DELTA * FACT1) / Q8) / Q8;
  const double hRST = RSTHRD * t2 * hBT * BEC * eurs, hT = 2.0 * BETA * (Q9 / Q8);
  const double FACT2 = Q4 * Q5 + B * t2 * (Q4 * Q9 + Q5), FACT3 = 2.0 * B * Q5 * Q9 + DELTA * FACT2;
  const double hTT = 4.0 * BETA * t * (2.0 * B / Q8 - ((Q9 / Q8) * FACT3) / Q8);
  double COMM = H + hRS + hRST + t2 * hT / 6.0 + 7.0 * t2 * t * hTT / 6.0;
  COMM = COMM - UU * hTT - VV * hT;
  *vcpbe = vclda + COMM;
}

/* g2g/pointxc/calc_ggaCS.h:36-57,127-149 */
static void gga_cs(double dens, const double* g, const double* h1, const double* h2, double* ex, double* ec,
                   double* y2a) {
  *ex = *ec = *y2a = 0.0;
  if (dens < 1e-18) return;
  double grad2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
  if (grad2 < DBL_MIN) grad2 = DBL_MIN;
  const double dgrad = sqrt(grad2);
  const double delgrad = (g[0] * g[0] * h1[0] + g[1] * g[1] * h1[1] + g[2] * g[2] * h1[2] +
                          2 * (g[0] * g[1] * h2[0] + g[0] * g[2] * h2[1] + g[1] * g[2] * h2[2])) /
                         dgrad;
  const double rlap = h1[0] + h1[1] + h1[2];
  double vx, vc;
  pbe_cs(dens, dgrad, delgrad, rlap, ex, &vx, ec, &vc);
  *y2a = vx + vc;
}

/* g2g/pointxc/calc_ggaCS.h:36-262 for iexch 4-8 (closed shell): exchange
 * Perdew 86 (4, 8) or Becke 88 (5-7); correlation Perdew 86 over the VWN-form
 * local part (4, 5), that local part alone (6) or Lee-Yang-Parr (7, 8). The
 * reference's constants, float literals included (FLT), and operation order. */
#define FLT(x) ((double)(float)(x))
static void gga_cs_other(double dens, const double* g, const double* h1, const double* h2, int iexch, double* ex,
                         double* ecout, double* y2a) {
  *ex = *ecout = *y2a = 0.0;
  if (dens < 1e-18) return;
  const double ALPHA = -0.738558766382022447, GL = 0.620350490899400087;
  const double VA1 = 0.03109205, VB1 = 3.72744, VC1 = 12.9352, VX0 = -0.10498, VQ = 6.15199066246304849;
  const double VA16 = 0.005182008333, VQ2 = 4.7309269;
  const double ALYP = 0.04918, BLYP = 0.132, CLYP = 0.2533, CLYP3 = 0.0844333333, DLYP = 0.349,
               DLYP3 = 0.116333333, CF = 2.87123400018819;
  const double B88 = 0.0042, ALF = 0.023266, BET = 7.389, GAM = 8.723, DEL = 0.472;
  const double y = cbrt(dens);
  double grad2 = g[0] * g[0] + g[1] * g[1] + g[2] * g[2];
  if (grad2 < DBL_MIN) grad2 = DBL_MIN;
  const double dgrad = sqrt(grad2);
  const double lap = h1[0] + h1[1] + h1[2];
  const double u0 = ((g[0] * g[0]) * h1[0] + 2.0 * g[0] * g[1] * h2[0] + 2.0 * g[1] * g[2] * h2[2] +
                     2.0 * g[0] * g[2] * h2[1] + (g[1] * g[1]) * h1[1] + (g[2] * g[2]) * h1[2]) /
                    dgrad;
  double v = 0.0;
  if (iexch == 4 || iexch == 8) {  // exchange: Perdew, PRB 33, 8800 (1986)
    const double dens2 = dens * dens;
    const double ckf = 3.0936677 * y;
    const double s = dgrad / (2.0 * ckf * dens);
    const double fx = 1.0 / 15.0;
    const double s2 = s * s, s3 = s * s * s, s4 = pow(s, 4);
    const double g0 = 1.0 + 1.296 * s2 + 14.0 * s4 + 0.2 * pow(s, 6);
    const double F = pow(g0, fx);
    *ex = ALPHA * F * y;
    const double t = lap / (dens * 4.0 * (ckf * ckf));
    const double u = u0 / (pow(2.0 * ckf, 3) * dens2);
    const double g2 = 2.592 * s + 56.0 * s3 + 1.2 * pow(s, 5);
    const double g3 = 2.592 + 56.0 * s2 + 1.2 * s4;
    const double g4 = 112.0 * s + 4.8 * s3;
    const double dF = fx * F / g0 * g2;
    const double dsF = fx * F / g0 * (-14.0 * fx * g3 * g2 / g0 + g4);
    v = ALPHA * y * (1.33333333333 * F - t / s * dF - (u - 1.3333333333 * s3) * dsF);
  } else {  // exchange: Becke, PRA 38, 3098 (1988)
    const double e0 = ALPHA * y;
    const double half = dens / 2.0;
    const double r13 = cbrt(half);
    const double r43 = cbrt(pow(half, 4));
    const double xs = dgrad / (2.0 * r43);
    const double ash = asinh(xs);
    const double dn = 1.0 + 6.0 * B88 * xs * ash;
    *ex = e0 + (-2.0 * B88 * r43 * xs * xs / (dn * dens));
    const double v0 = 1.33333333333333 * e0;
    const double fb = 1.0 / dn;
    const double xa1 = xs / sqrt(1.0 + xs * xs);
    const double dn1 = 1.0 + fb * (1.0 - 6.0 * B88 * xs * xa1);
    const double dn2 = 1.0 / (1.0 + xs * xs) + 2.0 * fb * (2.0 - 6.0 * B88 * xs * xa1);
    const double dn3 = ash * (1.0 + 2.0 * fb) + xa1 * dn2;
    const double d02 = lap / 2.0;
    const double de1 = 1.33333333333333 / (cbrt(pow(dens, 7)));
    const double c2 = cbrt(2.0);
    // d|grad|/da along each axis and the gradient of x_sigma
    const double dgx = (g[0] * h1[0] + g[1] * h2[0] + g[2] * h2[1]) / dgrad;
    const double gxx = c2 * (1.0 / (dens * y) * dgx - de1 * g[0] * dgrad);
    const double dgy = (g[0] * h2[0] + g[1] * h1[1] + g[2] * h2[2]) / dgrad;
    const double gxy = c2 * (1.0 / (dens * y) * dgy - de1 * g[1] * dgrad);
    const double dgz = (g[0] * h2[1] + g[1] * h2[2] + g[2] * h1[2]) / dgrad;
    const double gxz = c2 * (1.0 / (dens * y) * dgz - de1 * g[2] * dgrad);
    const double dn4 = 6.0 * B88 * fb * (g[0] / 2.0 * gxx + g[1] / 2.0 * gxy + g[2] / 2.0 * gxz);
    const double dn5 = 1.33333333333333 * r43 * r13 * xs * xs;
    const double tot2 = dn5 - d02 * dn1 + dn4 * dn3;
    v = v0 + (-B88 * fb / r43 * tot2);
  }
  if (iexch >= 4 && iexch <= 6) {  // correlation: VWN-form local part (+ Perdew, PRB 33, 8822 (1986))
    const double dens2 = dens * dens;
    const double rs = GL / y;
    const double x1 = sqrt(rs);
    const double Xx = rs + VB1 * x1 + VC1;
    const double Xxo = (VX0 * VX0) + VB1 * VX0 + VC1;
    const double t1 = 2.0 * x1 + VB1;
    const double t2 = log(Xx);
    const double t3 = atan(VQ / t1);
    const double t4 = VB1 * VX0 / Xxo;
    double ec = VA1 * (2.0 * log(x1) - t2 + 2.0 * VB1 / VQ * t3 -
                       t4 * (2.0 * log(x1 - VX0) - t2 + 2.0 * (VB1 + 2.0 * VX0) / VQ * t3));
    const double t5 = (VB1 * x1 + 2.0 * VC1) / x1;
    const double t6 = VX0 / Xxo;
    double vc = ec - VA16 * x1 *
                         (t5 / Xx - 4.0 * VB1 / ((t1 * t1) + (VQ * VQ2)) * (1.0 - t6 * (VB1 - 2.0 * VX0)) -
                          t4 * (2.0 / (x1 - VX0) - t1 / Xx));
    if (iexch != 6) {
      const double rs2 = rs * rs;
      const double cx1 = FLT(0.002568f) + ALF * rs + BET * rs2;
      const double cx2 = 1.0 + GAM * rs + DEL * rs2 + 1.0e4 * BET * (rs * rs * rs);
      const double C = 0.001667 + cx1 / cx2;
      const double cx3 = ALF + 2.0 * BET * rs;
      const double cx4 = GAM + 2.0 * DEL * rs + 3.0e4 * BET * rs2;
      double dC = cx3 / cx2 - cx1 / (cx2 * cx2) * cx4;
      dC = FLT(-0.333333333333333f) * dC * GL / (y * dens);
      const double phi = FLT(0.0008129082f) / C * dgrad / pow(dens, (double)(7.0f / 6.0f));
      const double ex_ = exp(-phi);
      const double ex0 = ex_ * C;
      ec = ec + ex0 * grad2 / (y * dens2);
      const double D1 = (2.0 - phi) * lap / dens;
      const double phi2 = phi * phi;
      double D2 = FLT(1.33333333333333333f) - FLT(3.666666666666666666f) * phi + FLT(1.166666666666666f) * phi2;
      D2 = D2 * grad2 / dens2;
      const double D3 = phi * (phi - 3.0) * u0 / (dens * dgrad);
      const double D4 = ex_ * grad2 / (y * dens) * (phi2 - phi - 1.0) * dC;
      vc = vc - 1.0 * (ex0 / y * (D1 - D2 + D3) - D4);
    }
    *ecout = ec;
    v = v + vc;
  } else {  // correlation: Lee, Yang, Parr, PRB 37, 785 (1988)
    const double rom13 = 1 / cbrt(dens);
    const double rom53 = cbrt(pow(dens, 5));
    const double ecro = exp(-CLYP * rom13);
    const double f1 = 1.0 / (1.0 + DLYP * rom13);
    const double tw = 0.125 * (grad2 / dens - lap);
    double term = (tw / 9.0 + lap / 18.0) - 2.0 * tw + CF * rom53;
    term = dens + BLYP * (rom13 * rom13) * ecro * term;
    *ecout = -ALYP * f1 * term / dens;
    const double hh1 = ecro / rom53;
    const double gg1 = f1 * hh1;
    const double tm1 = DLYP3 * (rom13 / dens);
    const double fp1 = tm1 * (f1 * f1);
    const double tm2 = FLT(-1.666666666f) + CLYP3 * rom13;
    const double hp1 = hh1 * tm2 / dens;
    const double gp1 = fp1 * hh1 + hp1 * f1;
    const double fp2 = tm1 * 2.0 * f1 * (fp1 - FLT(0.6666666666f) * f1 / dens);
    const double tm3 = FLT(1.6666666666f) - CLYP3 * FLT(1.3333333333f) * rom13;
    const double hp2 = hp1 * tm2 / dens + hh1 * tm3 / (dens * dens);
    const double gp2 = fp2 * hh1 + 2.0 * fp1 * hp1 + hp2 * f1;
    const double term3 = -ALYP * (fp1 * dens + f1) - ALYP * BLYP * CF * (gp1 * dens + (double)(8.0f / 3.0f) * gg1) * rom53;
    const double term4 = (gp2 * dens * grad2 + gp1 * (3.0 * grad2 + 2.0 * dens * lap) + 4.0 * gg1 * lap) * ALYP * BLYP / 4.0;
    const double term5 =
        (3.0 * gp2 * dens * grad2 + gp1 * (5.0 * grad2 + 6.0 * dens * lap) + 4.0 * gg1 * lap) * ALYP * BLYP / 72.0;
    v = v + (term3 - term4 - term5);
  }
  *y2a = v;
}


/* g2g/pointxc/pbeOS_exch.h:42-75 */
static void pbe_os_exch(double rho, double s, double u, double v, double* ex, double* vx) {
  const double UM = FL(0.2195149727645171f), UK = FL(0.804f), UL = FL(0.273028573090195f);
  const double exunif = FL(-0.738558766382022405884230032680836f) * cbrt(rho);
  const double s2 = s * s, s3 = s * s2, p0 = 1.0 + UL * s2, fxpbe = 1.0 + UK - UK / p0;
  *ex = exunif * fxpbe;
  const double Fs = 2.0 * UM / (p0 * p0), Fss = (-4.0 * UL * s * Fs) / p0;
  *vx = exunif * (F43 * fxpbe - (u - F43 * s3) * Fss - v * Fs);
}

/* g2g/pointxc/pbeOS_corr.h:63-251 */
static void pbe_os_corr(double rs, double zet, double t, double uu, double vv, double ww, double* ec, double* vca,
                        double* vcb, double* h, double* dvca, double* dvcb) {
  const double GAMMA = FL(0.03109069086965489503494086371273f), BETA = FL(0.06672455060314922f);
  const double DELTA = BETA / GAMMA, ETA = FL(0.000000000001f);
  const double rtrs = sqrt(rs);
  double EU, EURS, EP, EPRS, ALFM, ALFRSM;
  gcor(1, rtrs, &EU, &EURS);
  gcor(2, rtrs, &EP, &EPRS);
  gcor(3, rtrs, &ALFM, &ALFRSM);
  const double Z2 = zet * zet, Z4 = Z2 * Z2;
  const double GAM = pow(2.0, 4.0 / 3.0) - 2.0;
  const double F = (cbrt(pow(1.0 + zet, 4)) + cbrt(pow(1.0 - zet, 4)) - 2.0) / GAM;
  const double FZZ = 8.0 / (9.0 * GAM);
  *ec = EU * (1.0 - F * Z4) + EP * F * Z4 - ALFM * F * (1.0 - Z4) / FZZ;
  const double ECRS = EURS * (1.0 - F * Z4) + EPRS * F * Z4 - ALFRSM * F * (1.0 - Z4) / FZZ;
  const double FZ = F43 * (cbrt(1.0 + zet) - cbrt(1.0 - zet)) / GAM;
  const double ECZET = 4.0 * pow(zet, 3) * F * (EP - EU + ALFM / FZZ) + FZ * (Z4 * EP - Z4 * EU - (1.0 - Z4) * ALFM / FZZ);
  double COMM = *ec - rs * ECRS / 3.0 - zet * ECZET;
  *vca = COMM + ECZET;
  *vcb = COMM - ECZET;
  const double G = (cbrt(pow(1.0 + zet, 2)) + cbrt(pow(1.0 - zet, 2))) / 2.0, G3 = pow(G, 3);
  const double PON = -*ec / (G3 * GAMMA), B = DELTA / (exp(PON) - 1.0), B2 = B * B;
  const double T2 = t * t, T4 = T2 * T2, Q4 = 1.0 + B * T2, Q5 = 1.0 + B * T2 + B2 * T4;
  *h = G3 * (BETA / DELTA) * log(1.0 + DELTA * Q4 * T2 / Q5);
  const double G4 = G3 * G, T6 = T4 * T2, rsthrd = rs / 3.0;
  const double GZ = (pow(pow(1.0 + zet, 2) + ETA, (double)(-1.0f / 6.0f)) -
                     pow(pow(1.0 - zet, 2) + ETA, (double)(-1.0f / 6.0f))) / 3.0;
  const double FAC = DELTA / B + 1.0, BG = -3.0 * B2 * *ec * FAC / (BETA * G4), BEC = B2 * FAC / (BETA * G3);
  const double Q8 = pow(Q5, 2) + DELTA * Q4 * Q5 * T2, Q9 = 1.0 + 2.0 * B * T2;
  const double hB = -BETA * G3 * B * (T6 / Q8) * (2.0 + B * T2), hRS = -rsthrd * hB * BEC * ECRS;
  const double FACT0 = 2.0 * DELTA - 6.0 * B, FACT1 = Q5 * Q9 + Q4 * Q9 * Q9;
  const double hBT = 2.0 * BETA * G3 * T4 * ((Q4 * Q5 * FACT0 - DELTA * FACT1) / Q8) / Q8;
  const double hRST = rsthrd * T2 * hBT * BEC * ECRS;
  const double hz = 3.0 * GZ * *h / G + hB * (BG * GZ + BEC * ECZET);
  const double hT = 2.0 * BETA * G3 * Q9 / Q8;
  const double hZT = 3.0 * GZ * hT / G + hBT * (BG * GZ + BEC * ECZET);
  const double FACT2 = Q4 * Q5 + B * T2 * (Q4 * Q9 + Q5), FACT3 = 2.0 * B * Q5 * Q9 + DELTA * FACT2;
  const double hTT = 4.0 * BETA * G3 * t * (2.0 * B / Q8 - ((Q9 / Q8) * FACT3) / Q8);
  COMM = *h + hRS + hRST + T2 * hT / 6.0 + 7.0 * T2 * t * hTT / 6.0;
  const double PREF = hz - GZ * T2 * hT / G, FACT5 = GZ * (2.0 * hT + t * hTT) / G;
  COMM = COMM - PREF * zet - uu * hTT - vv * hT - ww * (hZT - FACT5);
  *dvca = COMM + PREF;
  *dvcb = COMM - PREF;
}

static void spin_terms(const double* g, const double* h1, const double* h2, double* dg, double* dl, double* lp) {
  *dg = sqrt(pow(g[0], 2) + pow(g[1], 2) + pow(g[2], 2));
  *dl = (pow(g[0], 2) * h1[0] + 2.0 * g[0] * g[1] * h2[0] + 2.0 * g[1] * g[2] * h2[2] + 2.0 * g[0] * g[2] * h2[1] +
         pow(g[1], 2) * h1[1] + pow(g[2], 2) * h1[2]) / *dg;
  *lp = h1[0] + h1[1] + h1[2];
}

/* g2g/pointxc/calc_ggaOS.h:11-109 with pbeOS_main.h:29-205 */
static void gga_os(double da, double db, const double* ga, const double* gb, const double* h1a, const double* h1b,
                   const double* h2a, const double* h2b, double* ex, double* ec, double* va, double* vb) {
  *ex = *ec = *va = *vb = 0.0;
  const double MIN = 1e-18;
  if (!((da > MIN) || (db > MIN))) return;
  const double PIF = FL(3.141592653589793238462643383279f), PI32 = FL(29.608813203268075856503472999628f);
  double dga, dla, lpa, dgb, dlb, lpb;
  spin_terms(ga, h1a, h2a, &dga, &dla, &lpa);
  spin_terms(gb, h1b, h2b, &dgb, &dlb, &lpb);
  double g[3], h1[3], h2[3];
  for (int k = 0; k < 3; k++) {
    g[k] = ga[k] + gb[k];
    h1[k] = h1a[k] + h1b[k];
    h2[k] = h2a[k] + h2b[k];
  }
  const double dgrad = sqrt(pow(g[0], 2) + pow(g[1], 2) + pow(g[2], 2));
  const double delgrad = (pow(g[0], 2) * h1[0] + pow(g[1], 2) * h1[1] + pow(g[2], 2) * h1[2] +
                          2.0 * g[0] * g[1] * h2[0] + 2.0 * g[1] * g[2] * h2[2] + 2.0 * g[0] * g[2] * h2[1]) / dgrad;
  double exs[2] = {0, 0}, vxs[2] = {0, 0};
  const double dd[2] = {da, db}, dgs[2] = {dga, dgb}, dls[2] = {dla, dlb}, lps[2] = {lpa, lpb};
  for (int sp = 0; sp < 2; sp++) {
    const double td = 2.0 * dd[sp];
    if (td > MIN) {
      const double td2 = td * td, fk = cbrt(PI32) * cbrt(td);
      const double tf = 2.0 * fk, tf2 = tf * tf, tf3 = tf * tf2;
      pbe_os_exch(td, (2.0 * dgs[sp]) / (td * tf), (4.0 * dls[sp]) / (td2 * tf3), (2.0 * lps[sp]) / (td * tf2),
                  &exs[sp], &vxs[sp]);
    }
  }
  const double rho = da + db;
  *ex = exs[0] * (da / rho) + exs[1] * (db / rho);
  *va = vxs[0];
  *vb = vxs[1];
  if (rho < (MIN * 1E5)) return;
  const double zet = (da - db) / rho, g1 = 1.0 + zet, g2 = 1.0 - zet;
  const double gg = (cbrt(g1 * g1) + cbrt(g2 * g2)) / 2.0;
  const double fk = cbrt(PI32) * cbrt(rho);
  const double rs = cbrt((9.0 * PIF) / 4.0) / fk;
  const double sk = sqrt(4.0 * fk / PIF), tks = 2.0 * sk * gg;
  const double t = dgrad / (tks * rho);
  const double uu = delgrad / (rho * rho * tks * tks * tks), vv = (lpa + lpb) / (rho * tks * tks);
  const double ww = ((dga * dga) - (dgb * dgb) - (zet * dgrad * dgrad)) / ((rho * rho) * (tks * tks));
  double c, vca, vcb, h, dvca, dvcb;
  pbe_os_corr(rs, zet, t, uu, vv, ww, &c, &vca, &vcb, &h, &dvca, &dvcb);
  *ec = c + h;
  *va = vxs[0] + vca + dvca;
  *vb = vxs[1] + vcb + dvcb;
}

/* ------------------------------------------------------------- basis values */
static const int comp_l[10][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0},
                                  {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}};

static double mono(const double* r, const int* l, const int* d) {
  /* d: derivative order per axis (0,1,2) of x^lx y^ly z^lz */
  double v = 1.0;
  for (int k = 0; k < 3; k++) {
    const int n = l[k], o = d[k];
    double f;
    if (o == 0) f = n == 0 ? 1.0 : (n == 1 ? r[k] : r[k] * r[k]);
    else if (o == 1) f = n == 0 ? 0.0 : (n == 1 ? 1.0 : 2.0 * r[k]);
    else f = n == 2 ? 2.0 : 0.0;
    v *= f;
  }
  return v;
}

/* g2g/cpu/functions.cpp:15-359: F, gradients (x,y,z), Hessian (xx,yy,zz) and (xy,xz,yz),
 * each stored point-major: v[k][p*m + i]. */
static void basis(const oracle_system* s, const group_t* g, int gga, double** v) {
  const int m = total_functions(g);
  const double nf = s->normalize ? 1.0 / sqrt(3) : 1.0;
  for (int q = 0; q < g->p.n; q++) {
    const pt_t* pt = &g->p.v[q];
    int ii = 0;
    for (int f = 0; f < g->nf; f++) {
      const int gf = g->funcs[f];
      const int a = s->nuc[gf];
      const double r[3] = {pt->x - s->x[a], pt->y - s->y[a], pt->z - s->z[a]};
      const double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      double t = 0, tg = 0, th = 0;
      for (int k = 0; k < s->ncont[gf]; k++) {
        const double aa = s->a[gf * MAXC + k], cc = s->c[gf * MAXC + k];
        if (aa * d2 > 70.0) continue;
        const double t0 = exp(-(aa * d2)) * cc;
        t += t0;
        tg += t0 * aa;
        th += t0 * (aa * aa);
      }
      const int type = gf < s->s_funcs ? 0 : (gf < s->s_funcs + 3 * s->p_funcs ? 1 : 2);
      const int c0 = type == 0 ? 0 : (type == 1 ? 1 : 4), nc = type == 0 ? 1 : (type == 1 ? 3 : 6);
      for (int cidx = 0; cidx < nc; cidx++, ii++) {
        const int* l = comp_l[c0 + cidx];
        const double sc = (type == 2 && (cidx == 0 || cidx == 2 || cidx == 5)) ? nf : 1.0;
        const int z0[3] = {0, 0, 0};
        const double P = mono(r, l, z0);
        const size_t o = (size_t)q * m + ii;
        v[0][o] = sc * P * t;
        if (!gga) continue;
        double Pa[3];
        for (int ax = 0; ax < 3; ax++) {
          int d[3] = {0, 0, 0};
          d[ax] = 1;
          Pa[ax] = mono(r, l, d);
          v[1 + ax][o] = sc * (Pa[ax] * t - 2.0 * r[ax] * P * tg);
        }
        static const int ha[6] = {0, 1, 2, 0, 0, 1}, hb[6] = {0, 1, 2, 1, 2, 2};
        for (int h = 0; h < 6; h++) {
          int d[3] = {0, 0, 0};
          d[ha[h]] += 1;
          d[hb[h]] += 1;
          const double Pab = mono(r, l, d);
          v[4 + h][o] = sc * (Pab * t - 2.0 * (r[hb[h]] * Pa[ha[h]] + r[ha[h]] * Pa[hb[h]] + (ha[h] == hb[h] ? P : 0.0)) * tg +
                              4.0 * r[ha[h]] * r[hb[h]] * P * th);
        }
      }
    }
  }
}

/* --------------------------------------------------------------- one group */
static long long pidx(int bi, int bj, int M) { /* bi <= bj, g2g/partition.cpp:64-66 */
  return (long long)bi * M - ((long long)bi * (bi - 1)) / 2 + (bj - bi);
}

/* density loops of g2g/cpu/iteration.cpp:90-176 (closed) and 366-467 (open) */
static void density_point(int m, int gga, const double* R, double* const* v, size_t row, double* q) {
  const double* fv = v[0] + row;
  if (!gga) {
    double pd = 0;
    for (int i = 0; i < m; i++) {
      double w = 0;
      for (int j = i; j < m; j++) w += R[(size_t)j * m + i] * fv[j];
      pd += fv[i] * w;
    }
    q[0] = pd;
    return;
  }
  const double *gx = v[1] + row, *gy = v[2] + row, *gz = v[3] + row, *hpx = v[4] + row, *hpy = v[5] + row,
               *hpz = v[6] + row, *hix = v[7] + row, *hiy = v[8] + row, *hiz = v[9] + row;
  double pd = 0, tdx = 0, tdy = 0, tdz = 0, d1x = 0, d1y = 0, d1z = 0, d2x = 0, d2y = 0, d2z = 0;
  for (int i = 0; i < m; i++) {
    double w = 0, w3x = 0, w3y = 0, w3z = 0, w1x = 0, w1y = 0, w1z = 0, w2x = 0, w2y = 0, w2z = 0;
    const double* rr = R + (size_t)i * m;
    for (int j = 0; j <= i; j++) {
      const double r = rr[j];
      w += fv[j] * r;
      w3x += gx[j] * r;
      w3y += gy[j] * r;
      w3z += gz[j] * r;
      w1x += hpx[j] * r;
      w1y += hpy[j] * r;
      w1z += hpz[j] * r;
      w2x += hix[j] * r;
      w2y += hiy[j] * r;
      w2z += hiz[j] * r;
    }
    const double F = fv[i];
    pd += F * w;
    tdx += gx[i] * w + w3x * F;
    d1x += gx[i] * w3x * 2 + hpx[i] * w + w1x * F;
    d2x += gx[i] * w3y + gy[i] * w3x + hix[i] * w + w2x * F;
    tdy += gy[i] * w + w3y * F;
    d1y += gy[i] * w3y * 2 + hpy[i] * w + w1y * F;
    d2y += gx[i] * w3z + gz[i] * w3x + hiy[i] * w + w2y * F;
    tdz += gz[i] * w + w3z * F;
    d1z += gz[i] * w3z * 2 + hpz[i] * w + w1z * F;
    d2z += gy[i] * w3z + gz[i] * w3y + hiz[i] * w + w2z * F;
  }
  q[0] = pd;
  q[1] = tdx; q[2] = tdy; q[3] = tdz;
  q[4] = d1x; q[5] = d1y; q[6] = d1z;
  q[7] = d2x; q[8] = d2y; q[9] = d2z;
}

/* One group's E_xc; with Ka, its Kohn-Sham contributions (+=); with frc
 * (natoms x 3, [atom * 3 + axis]), its XC forces (+=) instead, the
 * reference's force loop g2g/cpu/iteration.cpp:213-267 (open: 496-563). */
static double solve_group(const oracle_system* s, const group_t* g, const double* Pa, const double* Pb, double* Ka,
                          double* Kb, double* frc) {
  const int m = total_functions(g), n = g->p.n, gga = s->iexch > 3;
  const int nk = (gga || frc) ? 10 : 1;
  int* gl = (int*)malloc(sizeof(int) * (size_t)m);
  for (int f = 0, ii = 0; f < g->nf; f++) {
    const int gf = g->funcs[f];
    const int nc = gf < s->s_funcs ? 1 : (gf < s->s_funcs + 3 * s->p_funcs ? 3 : 6);
    for (int k = 0; k < nc; k++) gl[ii++] = gf + k;
  }
  double* v[10] = {0};
  for (int k = 0; k < nk; k++) v[k] = (double*)calloc((size_t)n * m, sizeof(double));
  basis(s, g, gga || frc, v);
  const int nsp = s->open ? 2 : 1;
  double* R[2] = {0, 0};
  for (int sp = 0; sp < nsp; sp++) {
    const double* P = sp == 0 ? Pa : Pb;
    R[sp] = (double*)malloc(sizeof(double) * (size_t)m * m);
    for (int i = 0; i < m; i++)
      for (int j = i; j < m; j++) {
        const double val = P[pidx(gl[i], gl[j], s->M)];
        R[sp][(size_t)i * m + j] = R[sp][(size_t)j * m + i] = val;
      }
  }
  double* fa = (double*)malloc(sizeof(double) * (size_t)n);
  double* fb = s->open ? (double*)malloc(sizeof(double) * (size_t)n) : NULL;
  double energy = 0.0;
  for (int p = 0; p < n; p++) {
    const size_t row = (size_t)p * m;
    const double w = g->p.v[p].w;
    double qa[10] = {0}, qb[10] = {0};
    density_point(m, gga, R[0], v, row, qa);
    if (s->open) {
      density_point(m, gga, R[1], v, row, qb);
      double ex = 0, ec = 0, va = 0, vb = 0;
      if (gga) gga_os(qa[0], qb[0], qa + 1, qb + 1, qa + 4, qb + 4, qa + 7, qb + 7, &ex, &ec, &va, &vb);
      energy += ((qa[0] + qb[0]) * w) * (ex + ec);
      fa[p] = w * va;
      fb[p] = w * vb;
    } else {
      double ex, ec, y2a;
      if (gga && s->iexch != 9)
        gga_cs_other(qa[0], qa + 1, qa + 4, qa + 7, s->iexch, &ex, &ec, &y2a);
      else if (gga)
        gga_cs(qa[0], qa + 1, qa + 4, qa + 7, &ex, &ec, &y2a);
      else
        lda(qa[0], s->iexch, &ex, &ec, &y2a);
      energy += (qa[0] * w) * (ex + ec);
      fa[p] = w * y2a;
    }
  }
  if (frc) {
    /* per point: dd[atom] = -sum over the atom's functions ii of w_ii grad F_ii,
     * w_ii = sum_j R_j,ii F_j (x 2 for j = ii); forces[atom] += dd * factor over
     * the points in order, per spin, and the spins added at the end */
    const int nsp2 = s->open ? 2 : 1;
    double* dd = (double*)calloc((size_t)s->natoms * 3, sizeof(double));
    double* acc = (double*)calloc((size_t)s->natoms * 3 * 2, sizeof(double));
    for (int sp = 0; sp < nsp2; sp++) {
      const double* Rs = R[sp];
      const double* fac = sp == 0 ? fa : fb;
      double* ac = acc + (size_t)sp * s->natoms * 3;
      for (int p = 0; p < n; p++) {
        const double* fv = v[0] + (size_t)p * m;
        for (int f = 0, ii = 0; f < g->nf; f++) {
          const int gf = g->funcs[f];
          const int nc = gf < s->s_funcs ? 1 : (gf < s->s_funcs + 3 * s->p_funcs ? 3 : 6);
          const int atom = s->nuc[gf];
          double tx = 0.0, ty = 0.0, tz = 0.0;
          for (int k = 0; k < nc; k++, ii++) {
            double w = 0.0;
            for (int j = 0; j < m; j++) w += Rs[(size_t)j * m + ii] * fv[j] * (ii == j ? 2 : 1);
            const size_t o = (size_t)p * m + ii;
            tx -= w * v[1][o];
            ty -= w * v[2][o];
            tz -= w * v[3][o];
          }
          dd[atom * 3 + 0] += tx;
          dd[atom * 3 + 1] += ty;
          dd[atom * 3 + 2] += tz;
        }
        for (int f = 0; f < g->nf; f++) {  /* each atom of the group once, then cleared */
          const int atom = s->nuc[g->funcs[f]];
          for (int x = 0; x < 3; x++) {
            ac[atom * 3 + x] += dd[atom * 3 + x] * fac[p];
            dd[atom * 3 + x] = 0.0;
          }
        }
      }
    }
    for (int f = 0; f < g->nf; f++) {  /* every atom of the group once: its sum, then cleared */
      const int atom = s->nuc[g->funcs[f]];
      for (int x = 0; x < 3; x++) {
        frc[atom * 3 + x] += acc[atom * 3 + x] + (s->open ? acc[(size_t)s->natoms * 3 + atom * 3 + x] : 0.0);
        acc[atom * 3 + x] = 0.0;
        if (s->open) acc[(size_t)s->natoms * 3 + atom * 3 + x] = 0.0;
      }
    }
    free(dd);
    free(acc);
  }
  /* Kohn-Sham accumulation: g2g/cpu/iteration.cpp:270-291 (open: 581-604) */
  for (int i = 0; i < m && Ka; i++)
    for (int j = i; j < m; j++) {
      double ra = 0.0, rb = 0.0;
      for (int p = 0; p < n; p++) {
        const double fij = v[0][(size_t)p * m + i] * v[0][(size_t)p * m + j];
        ra += fij * fa[p];
        if (s->open) rb += fij * fb[p];
      }
      const long long o = pidx(gl[i], gl[j], s->M);
      Ka[o] += ra;
      if (s->open) Kb[o] += rb;
    }
  for (int k = 0; k < nk; k++) free(v[k]);
  free(R[0]);
  free(R[1]);
  free(fa);
  free(fb);
  free(gl);
  return energy;
}

static int solve_groups_list(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                             double* fock, double* fockb, double* energy, long long* npoints, long long* ngroups,
                             int first, int stride, const int* ids, int nids, double* forces);

int oracle_solve_forces(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                        double* forces, double* energy, long long* npoints, long long* ngroups) {
  if (!forces) return -1;
  return solve_groups_list(s, rho, rho_a, rho_b, NULL, NULL, energy, npoints, ngroups, 0, 1, NULL, 0, forces);
}

int oracle_solve_sample(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                        double* fock, double* fockb, double* energy, long long* npoints, long long* ngroups,
                        int first, int stride) {
  return solve_groups_list(s, rho, rho_a, rho_b, fock, fockb, energy, npoints, ngroups, first, stride, NULL, 0, NULL);
}

int oracle_solve_subset(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                        double* fock, double* fockb, double* energy, long long* npoints, long long* ngroups,
                        const int* group_ids, int nids) {
  if (!group_ids || nids < 0) return -1;
  return solve_groups_list(s, rho, rho_a, rho_b, fock, fockb, energy, npoints, ngroups, 0, 1, group_ids, nids, NULL);
}

/* Groups first, first + stride, ... or, when ids != NULL, exactly ids[0 .. nids) (the
 * partition's order: cubes, then spheres, each sorted by cost). With forces
 * (natoms x 3 column-major, leading dimension natoms), XC forces are added
 * there and no Kohn-Sham contributions are formed (fock may be NULL). */
static int solve_groups_list(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b,
                             double* fock, double* fockb, double* energy, long long* npoints, long long* ngroups,
                             int first, int stride, const int* ids, int nids, double* forces) {
  if (!s || s->natoms <= 0 || s->M <= 0 || stride <= 0) return -1;
  if (s->open && (!rho_a || !rho_b || (!forces && !fockb))) return -2;
  if (!forces && !fock) return -1;
  int ng = 0;
  group_t* gs = build_groups(s, &ng);
  int* list = (int*)malloc(sizeof(int) * ((size_t)ng + 1));
  int nl = 0;
  if (ids) {
    for (int k = 0; k < nids; k++)
      if (ids[k] >= 0 && ids[k] < ng) list[nl++] = ids[k];
  } else {
    for (int gi = first; gi < ng; gi += stride) list[nl++] = gi;
  }
  const size_t np = (size_t)s->M * (s->M + 1) / 2;
  double* eg = (double*)calloc((size_t)ng + 1, sizeof(double));
  int nth = 1;
#ifdef _OPENMP
#pragma omp parallel
#pragma omp single
  nth = omp_get_num_threads();
#endif
  double* Ka = forces ? NULL : (double*)calloc(np * (size_t)nth, sizeof(double));
  double* Kb = (s->open && !forces) ? (double*)calloc(np * (size_t)nth, sizeof(double)) : NULL;
  double* Fr = forces ? (double*)calloc((size_t)s->natoms * 3 * (size_t)nth, sizeof(double)) : NULL;
  long long pts = 0, used = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : pts, used)
  for (int li = 0; li < nl; li++) {
    const int gi = list[li];
    int t = 0;
#ifdef _OPENMP
    t = omp_get_thread_num();
#endif
    eg[gi] = solve_group(s, &gs[gi], s->open ? rho_a : rho, rho_b, Ka ? Ka + np * (size_t)t : NULL,
                         Kb ? Kb + np * (size_t)t : NULL, Fr ? Fr + (size_t)s->natoms * 3 * (size_t)t : NULL);
    pts += gs[gi].p.n;
    used++;
  }
  double e = 0.0;
  for (int gi = 0; gi < ng; gi++) e += eg[gi];
  for (int t = 0; t < nth && Ka; t++)
    for (size_t i = 0; i < np; i++) {
      fock[i] += Ka[np * (size_t)t + i];
      if (s->open) fockb[i] += Kb[np * (size_t)t + i];
    }
  for (int t = 0; t < nth && Fr; t++)
    for (int a = 0; a < s->natoms; a++)
      for (int x = 0; x < 3; x++) forces[a + (size_t)s->natoms * x] += Fr[((size_t)t * s->natoms + a) * 3 + x];
  *energy = e;
  if (npoints) *npoints = pts;
  if (ngroups) *ngroups = used;
  for (int gi = 0; gi < ng; gi++) {
    free(gs[gi].p.v);
    free(gs[gi].funcs);
    free(gs[gi].nucs);
  }
  free(gs);
  free(eg);
  free(Ka);
  free(Kb);
  free(Fr);
  free(list);
  return 0;
}

int oracle_solve(const oracle_system* s, const double* rho, const double* rho_a, const double* rho_b, double* fock,
                 double* fockb, double* energy, long long* npoints, long long* ngroups) {
  return oracle_solve_sample(s, rho, rho_a, rho_b, fock, fockb, energy, npoints, ngroups, 0, 1);
}
