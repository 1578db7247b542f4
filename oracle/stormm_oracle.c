/*
 * FP64 CPU restatement of STORMM's implicit-solvent molecular mechanics for one molecule.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see stormm_oracle.h).  Plain loops
 * over atom pairs in double precision; the formulas follow STORMM's CPU evaluators, cited per
 * function.  Summation order differs from STORMM's tiled loops, which changes results only at
 * the level of double-precision rounding.
 */
#include "stormm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Constants/generalized_born.h:21-44, 114-126; Constants/scaling.h:30 */
static const double GB_TAYLOR_A = 0.33333333333333333333;
static const double GB_TAYLOR_B = 0.4;
static const double GB_TAYLOR_C = 0.42857142857142857143;
static const double GB_TAYLOR_D = 0.44444444444444444444;
static const double GB_TAYLOR_DD = 0.45454545454545454545;
static const double GB_TAYLOR_E = 1.33333333333333333333;
static const double GB_TAYLOR_F = 2.4;
static const double GB_TAYLOR_G = 3.42857142857142857143;
static const double GB_TAYLOR_H = 4.44444444444444444444;
static const double GB_TAYLOR_HH = 5.45454545454545454545;
static const double GB_RADII_OFFSET = 0.09;
static const double GB_KSCALE = 0.73;
static const double GB_SALT_KAPPA = 0.10806;
static const double VERYTINY = 1.0e-12;
/* Constants/symbol_values.h:72,81 */
static const double ASYMPTOTIC_TO_ONE = 0.99999904632568359375;
static const double INV_ONE_MINUS_ASYMPTOTE = 1048576.0;
/* Constants/symbol_values.h:75, the threshold for the arcsine route of Math/rounding.tpp:25-60 */
static const double NEAR_TO_ONE = 0.999999992549419403076171875;

static double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

static void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* ---------------------------------------------------------------------------------------------
 * Valence terms (Potential/valence_potential.tpp)
 * ------------------------------------------------------------------------------------------- */

/* evalHarmonicStretch, valence_potential.tpp:9-97 */
static double bond_term(const double* c, double* f, int i, int j, double k, double r0) {
  double d[3];
  for (int a = 0; a < 3; a++) d[a] = c[3 * j + a] - c[3 * i + a];
  const double r = sqrt(dot3(d, d));
  const double dl = r - r0;
  if (f) {
    const double fmag = 2.0 * k * dl / r;
    for (int a = 0; a < 3; a++) {
      f[3 * i + a] += fmag * d[a];
      f[3 * j + a] -= fmag * d[a];
    }
  }
  return k * dl * dl;
}

/* evalHarmonicBend, valence_potential.tpp:170-288 */
static double angle_term(const double* c, double* f, int i, int j, int k, double keq,
                         double theta0) {
  double ba[3], bc[3];
  for (int a = 0; a < 3; a++) {
    ba[a] = c[3 * i + a] - c[3 * j + a];
    bc[a] = c[3 * k + a] - c[3 * j + a];
  }
  const double mgba = dot3(ba, ba);
  const double mgbc = dot3(bc, bc);
  const double invbabc = 1.0 / sqrt(mgba * mgbc);
  double costheta = dot3(ba, bc) * invbabc;
  costheta = (costheta < -1.0) ? -1.0 : (costheta > 1.0) ? 1.0 : costheta;
  const double theta = acos(costheta);
  const double dtheta = theta - theta0;
  if (f) {
    const double dA = -2.0 * keq * dtheta / sqrt(1.0 - costheta * costheta);
    const double sqba = dA / mgba;
    const double sqbc = dA / mgbc;
    const double mbabc = dA * invbabc;
    for (int a = 0; a < 3; a++) {
      const double adf = bc[a] * mbabc - costheta * ba[a] * sqba;
      const double cdf = ba[a] * mbabc - costheta * bc[a] * sqbc;
      f[3 * i + a] -= adf;
      f[3 * j + a] += adf + cdf;
      f[3 * k + a] -= cdf;
    }
  }
  return keq * dtheta * dtheta;
}

/* Signed dihedral angle with the arcsine route near 0 / pi, Math/rounding.tpp:25-60 */
static double signed_dihedral(double costheta, const double* crabbc, const double* crbccd,
                              const double* bc, const double* scr) {
  const double sgn = (dot3(scr, bc) > 0.0) ? 1.0 : -1.0;
  if (fabs(costheta) >= NEAR_TO_ONE) {
    const double ia = 1.0 / sqrt(dot3(crabbc, crabbc));
    const double ib = 1.0 / sqrt(dot3(crbccd, crbccd));
    double rd[3];
    for (int a = 0; a < 3; a++) rd[a] = crbccd[a] * ib - crabbc[a] * ia;
    double rs = sqrt(dot3(rd, rd));
    if (fabs(rs) > 1.0) {
      for (int a = 0; a < 3; a++) rd[a] = crbccd[a] * ib + crabbc[a] * ia;
      rs = 3.14159265358979323846 - sqrt(dot3(rd, rd));
    }
    return sgn * rs;
  }
  return sgn * acos(costheta);
}

/* evalDihedralTwist (cosine style), valence_potential.tpp:359-578 */
static double dihedral_term(const double* c, double* f, int i, int j, int k, int l, double amp,
                            double phase, double freq) {
  double ab[3], bc[3], cd[3], crabbc[3], crbccd[3], scr[3];
  for (int a = 0; a < 3; a++) {
    ab[a] = c[3 * j + a] - c[3 * i + a];
    bc[a] = c[3 * k + a] - c[3 * j + a];
    cd[a] = c[3 * l + a] - c[3 * k + a];
  }
  cross3(ab, bc, crabbc);
  cross3(bc, cd, crbccd);
  double costheta = dot3(crabbc, crbccd) / sqrt(dot3(crabbc, crabbc) * dot3(crbccd, crbccd));
  cross3(crabbc, crbccd, scr);
  costheta = (costheta < -1.0) ? -1.0 : (costheta > 1.0) ? 1.0 : costheta;
  const double theta = signed_dihedral(costheta, crabbc, crbccd, bc, scr);
  const double sangle = freq * theta - phase;
  if (f) {
    const double fr = amp * freq * sin(sangle);
    const double mgab = sqrt(dot3(ab, ab));
    const double mgbc = sqrt(dot3(bc, bc));
    const double mgcd = sqrt(dot3(cd, cd));
    const double invab = 1.0 / mgab;
    const double invbc = 1.0 / mgbc;
    const double invcd = 1.0 / mgcd;
    const double cosb = -dot3(ab, bc) * invab * invbc;
    const double cosc = -dot3(bc, cd) * invbc * invcd;
    const double isinb2 = (cosb * cosb < ASYMPTOTIC_TO_ONE) ? fr / (1.0 - cosb * cosb) :
                                                               fr * INV_ONE_MINUS_ASYMPTOTE;
    const double isinc2 = (cosc * cosc < ASYMPTOTIC_TO_ONE) ? fr / (1.0 - cosc * cosc) :
                                                               fr * INV_ONE_MINUS_ASYMPTOTE;
    const double invabc = invab * invbc;
    const double invbcd = invbc * invcd;
    for (int a = 0; a < 3; a++) {
      crabbc[a] *= invabc;
      crbccd[a] *= invbcd;
    }
    const double fa = -invab * isinb2;
    const double fb1 = (mgbc - mgab * cosb) * invabc * isinb2;
    const double fb2 = cosc * invbc * isinc2;
    const double fd = -invcd * isinc2;
    for (int a = 0; a < 3; a++) {
      const double fi = crabbc[a] * fa;
      const double fj = fb1 * crabbc[a] - fb2 * crbccd[a];
      const double fl = -fd * crbccd[a];
      f[3 * i + a] += fi;
      f[3 * j + a] += fj;
      f[3 * k + a] -= fi + fj + fl;
      f[3 * l + a] += fl;
    }
  }
  return amp * (1.0 + cos(sangle));
}

/* ---------------------------------------------------------------------------------------------
 * Softened cores for clash damping, Potential/soft_core_potentials.tpp:30-52 (quadratic
 * Coulomb core below an absolute distance) and :140-180 (quartic Lennard-Jones core below a
 * ratio of the pair's sigma = (A/B)^(1/6), zero where B <= 1e-6).  Each adds the pair's energy
 * to *e and its force factor (force = fmag * displacement) to *fmag.
 * ------------------------------------------------------------------------------------------- */
static const double SOFT_CORE_TINY = 1.0e-10;

static void quadratic_core_coulomb(double r, double cd, double qiqj, double* e, double* fmag) {
  if (r < cd) {
    const double a = -0.5 / (cd * cd * (cd + 1.0));
    const double b = 1.0 / cd - a * (cd + 1.0) * (cd + 1.0);
    *e += qiqj * (a * (r + 1.0) * (r + 1.0) + b);
    if (r > SOFT_CORE_TINY) *fmag += qiqj * (2.0 * a + 2.0 * a / r);
  }
  else {
    const double invr = 1.0 / r;
    *e += qiqj * invr;
    *fmag -= qiqj * invr * invr * invr;
  }
}

static void quartic_core_lj(double r, double ratio, double lja, double ljb, double* e,
                            double* fmag) {
  const double sigma = (ljb > 1.0e-6) ? sqrt(cbrt(lja / ljb)) : 0.0;
  const double rl = ratio * sigma;
  if (r < rl) {
    const double il = 1.0 / rl;
    const double il6 = il * il * il * il * il * il;
    const double a = ((6.0 * ljb - 12.0 * lja * il6) * il * il6) /
                     ((((4.0 * rl + 12.0) * rl + 12.0) * rl) + 4.0);
    const double rlp = rl + 1.0;
    const double b = (lja * il6 - ljb) * il6 - a * rlp * rlp * rlp * rlp;
    const double rp = r + 1.0;
    const double a3 = a * rp * rp * rp;
    *e += a3 * rp + b;
    if (r > SOFT_CORE_TINY) *fmag += 4.0 * a3 / r;
  }
  else {
    const double invr2 = 1.0 / (r * r);
    const double invr4 = invr2 * invr2;
    *e += lja * invr4 * invr4 * invr4 - ljb * invr4 * invr2;
    *fmag += (6.0 * ljb - 12.0 * lja * invr4 * invr2) * invr4 * invr4;
  }
}

/* evalAttenuated14Pair, valence_potential.tpp:1288-1420; clash softening when cd > 0 or
 * ratio > 0 */
static void pair14_term(const orc_system* s, const double* c, double* f, int i, int l,
                        double scee, double scnb, double cd, double ratio, double* e_elec,
                        double* e_vdw) {
  double d[3];
  for (int a = 0; a < 3; a++) d[a] = c[3 * l + a] - c[3 * i + a];
  const int t = s->lj_idx[i] * s->n_lj_types + s->lj_idx[l];
  const double lja = s->lja14[t] / scnb;
  const double ljb = s->ljb14[t] / scnb;
  const double qiqj = s->coulomb_constant * s->charge[i] * s->charge[l] / scee;
  double fmag = 0.0;
  if (cd > 0.0 || ratio > 0.0) {
    const double r = sqrt(dot3(d, d));
    quadratic_core_coulomb(r, cd, qiqj, e_elec, &fmag);
    quartic_core_lj(r, ratio, lja, ljb, e_vdw, &fmag);
  }
  else {
    const double invr2 = 1.0 / dot3(d, d);
    const double invr = sqrt(invr2);
    const double invr4 = invr2 * invr2;
    *e_elec += qiqj * invr;
    *e_vdw += lja * invr4 * invr4 * invr4 - ljb * invr4 * invr2;
    fmag = -(qiqj * invr * invr2) + (6.0 * ljb - 12.0 * lja * invr4 * invr2) * invr4 * invr4;
  }
  if (f) {
    for (int a = 0; a < 3; a++) {
      f[3 * i + a] += fmag * d[a];
      f[3 * l + a] -= fmag * d[a];
    }
  }
}

/* ---------------------------------------------------------------------------------------------
 * Coulomb + Lennard-Jones over non-excluded pairs, nonbonded_potential.tpp:8-425
 * ------------------------------------------------------------------------------------------- */
static void nonbonded_terms(const orc_system* s, const double* c, double* f, double cd,
                            double ratio, double* e_elec, double* e_vdw) {
  const int soft = (cd > 0.0 || ratio > 0.0);
  const int n = s->natom;
  char* excl = (char*)calloc((size_t)n, 1);
  for (int i = 0; i < n; i++) {
    for (int e = s->excl_bounds[i]; e < s->excl_bounds[i + 1]; e++) {
      excl[s->excl_list[e]] = 1;
    }
    const double qi = s->coulomb_constant * s->charge[i];
    const int ti = s->lj_idx[i];
    for (int j = i + 1; j < n; j++) {
      if (excl[j]) continue;
      double d[3];
      for (int a = 0; a < 3; a++) d[a] = c[3 * j + a] - c[3 * i + a];
      const double invr2 = 1.0 / dot3(d, d);
      const double invr = sqrt(invr2);
      const double invr4 = invr2 * invr2;
      const double qiqj = qi * s->charge[j];
      const int t = s->lj_idx[j] * s->n_lj_types + ti;
      const double lja = s->lja[t];
      const double ljb = s->ljb[t];
      if (soft) {
        /* clash-mitigated loops, nonbonded_potential.tpp:108-175 */
        const double r = sqrt(dot3(d, d));
        double fmag = 0.0;
        quadratic_core_coulomb(r, cd, qiqj, e_elec, &fmag);
        quartic_core_lj(r, ratio, lja, ljb, e_vdw, &fmag);
        if (f) {
          for (int a = 0; a < 3; a++) {
            f[3 * i + a] += fmag * d[a];
            f[3 * j + a] -= fmag * d[a];
          }
        }
        continue;
      }
      *e_elec += qiqj * invr;
      *e_vdw += (lja * invr4 * invr4 - ljb * invr2) * invr4;
      if (f) {
        const double fmag = -(qiqj * invr * invr2) +
                            (6.0 * ljb - 12.0 * lja * invr4 * invr2) * invr4 * invr4;
        for (int a = 0; a < 3; a++) {
          f[3 * i + a] += fmag * d[a];
          f[3 * j + a] -= fmag * d[a];
        }
      }
    }
    for (int e = s->excl_bounds[i]; e < s->excl_bounds[i + 1]; e++) {
      excl[s->excl_list[e]] = 0;
    }
  }
  free(excl);
}

/* ---------------------------------------------------------------------------------------------
 * Generalized Born, nonbonded_potential.tpp:448-1294
 * ------------------------------------------------------------------------------------------- */

/* Descreening of an atom with offset radius rho by a neighbour of screened radius sj at
 * distance r (the Hawkins-Cramer-Truhlar integral), nonbonded_potential.tpp:589-640 */
static double hct_integral(double r, double rho, double sj) {
  const double r2 = r * r;
  const double invr = 1.0 / r;
  const double sj2 = sj * sj;
  if (r > 4.0 * sj) {
    const double invr2 = invr * invr;
    const double t = sj2 * invr2;
    const double dumbo = GB_TAYLOR_A + t * (GB_TAYLOR_B + t * (GB_TAYLOR_C +
                                                               t * (GB_TAYLOR_D + t * GB_TAYLOR_DD)));
    return sj * t * invr2 * dumbo;
  }
  if (r > rho + sj) {
    return 0.5 * (sj / (r2 - sj2) + 0.5 * invr * log((r - sj) / (r + sj)));
  }
  if (r > fabs(rho - sj)) {
    const double inv_rho = 1.0 / rho;
    const double theta = 0.5 * inv_rho * invr * (r2 + rho * rho - sj2);
    const double uij = 1.0 / (r + sj);
    return 0.25 * (inv_rho * (2.0 - theta) - uij + invr * log(rho * uij));
  }
  if (rho < sj) {
    return 0.5 * (sj / (r2 - sj2) + 2.0 / rho + 0.5 * invr * log((sj - r) / (sj + r)));
  }
  return 0.0;
}

/* Radial derivative factor of hct_integral (divided by r), nonbonded_potential.tpp:1116-1165 */
static double hct_derivative(double r, double rho, double sj) {
  const double r2 = r * r;
  const double invr = 1.0 / r;
  const double invr2 = invr * invr;
  const double sj2 = sj * sj;
  if (r > 4.0 * sj) {
    const double t = sj2 * invr2;
    const double dumbo = GB_TAYLOR_E + t * (GB_TAYLOR_F + t * (GB_TAYLOR_G +
                                                               t * (GB_TAYLOR_H + t * GB_TAYLOR_HH)));
    return t * sj * invr2 * invr2 * dumbo;
  }
  if (r > rho + sj) {
    const double temp1 = 1.0 / (r2 - sj2);
    return temp1 * sj * (-0.5 * invr2 + temp1) + 0.25 * invr * invr2 * log((r - sj) / (r + sj));
  }
  if (r > fabs(rho - sj)) {
    const double temp1 = 1.0 / (r + sj);
    const double invr3 = invr2 * invr;
    const double inv_rho = 1.0 / rho;
    return -0.25 * (-0.5 * (r2 - rho * rho + sj2) * invr3 * inv_rho * inv_rho +
                    invr * temp1 * (temp1 - invr) - invr3 * log(rho * temp1));
  }
  if (rho < sj) {
    const double temp1 = 1.0 / (r2 - sj2);
    return -0.5 * (sj * invr2 * temp1 - 2.0 * sj * temp1 * temp1 -
                   0.5 * invr2 * invr * log((sj - r) / (sj + r)));
  }
  return 0.0;
}

/* Neck GB (Mongan's union of spheres, nonbonded_potential.tpp:678-702): the amount psi_i
 * decreases by from neighbour j at distance r, and its radial derivative divided by r, both
 * from the tables of maximum separation and maximum value for the pair of neck indices */
static double neck_term(const orc_system* s, int i, int j, double r, double scale,
                        double* deriv) {
  const int t = s->neck_table_size * s->neck_idx[j] + s->neck_idx[i];
  const double m = r - s->neck_max_sep[t];
  const double m2 = m * m;
  const double den = 1.0 + m2 + 0.3 * m2 * m2 * m2;
  *deriv = ((2.0 * m + 1.8 * m2 * m2 * m) * s->neck_max_val[t] * scale) / (den * den * r);
  return scale * s->neck_max_val[t] / den;
}

static int is_neck(int igb) { return igb == ORC_GB_NECK || igb == ORC_GB_NECK2; }

/* Baseline radius offset and neck scale of the model (energy_abstracts.tpp:9-31) */
static double gb_offset(int igb) { return (igb == ORC_GB_NECK2) ? 0.195141 : GB_RADII_OFFSET; }
static double neck_scale(int igb) { return (igb == ORC_GB_NECK2) ? 0.826836 : 0.361825; }

static void gb_terms(const orc_system* s, const double* c, double* f, double* e_gb,
                     double* psi_out, double* radii_out, double* sdeijda_out) {
  const int n = s->natom;
  const double offset = gb_offset(s->igb);
  const int neck = is_neck(s->igb);
  const double nscale = neck_scale(s->igb);
  double* psi = (double*)calloc((size_t)n, sizeof(double));
  double* rad = (double*)calloc((size_t)n, sizeof(double));
  double* sde = (double*)calloc((size_t)n, sizeof(double));
  const double kappa = (s->saltcon > 1.0e-8) ? sqrt(GB_SALT_KAPPA * s->saltcon) : 0.0;
  const double diel = s->dielectric;

  /* Pass 1: Born radius descreening sums (psi accumulates the negated integrals) */
  for (int i = 0; i < n; i++) {
    const double rho_i = s->pb_radii[i] - offset;
    const double si = s->gb_screen[i] * rho_i;
    for (int j = i + 1; j < n; j++) {
      const double rho_j = s->pb_radii[j] - offset;
      const double sj = s->gb_screen[j] * rho_j;
      double d[3];
      for (int a = 0; a < 3; a++) d[a] = c[3 * i + a] - c[3 * j + a];
      const double r = sqrt(dot3(d, d));
      psi[i] -= hct_integral(r, rho_i, sj);
      psi[j] -= hct_integral(r, rho_j, si);
      if (neck && r < rho_i + rho_j + 2.0 * offset + s->neck_cut) {
        double unused;
        psi[i] -= neck_term(s, i, j, r, nscale, &unused);
        psi[j] -= neck_term(s, j, i, r, nscale, &unused);
      }
    }
  }

  /* Effective radii, nonbonded_potential.tpp:730-781 */
  for (int i = 0; i < n; i++) {
    const double rho = s->pb_radii[i] - offset;
    if (s->igb == ORC_GB_HCT) {
      double egbi = 1.0 / (1.0 / rho + psi[i]);
      if (egbi < 0.0) egbi = 30.0;
      rad[i] = egbi;
    }
    else {
      const double fipsi = psi[i] * (-rho);
      rad[i] = 1.0 / (1.0 / rho - tanh((s->gb_alpha[i] - s->gb_beta[i] * fipsi +
                                        s->gb_gamma[i] * fipsi * fipsi) * fipsi) /
                                   s->pb_radii[i]);
    }
  }

  /* Self terms, nonbonded_potential.tpp:784-805 */
  double egb = 0.0;
  for (int i = 0; i < n; i++) {
    const double q = s->charge[i];
    const double ri = rad[i];
    const double expmkf = exp(-GB_KSCALE * kappa * ri) / diel;
    const double dielfac = 1.0 - expmkf;
    const double atmq2h = 0.5 * q * q * s->coulomb_constant;
    const double atmqd2h = atmq2h * dielfac;
    egb += -atmqd2h / ri;
    sde[i] = atmqd2h - GB_KSCALE * kappa * atmq2h * expmkf * ri;
  }

  /* Pass 2: pair energies and direct forces, nonbonded_potential.tpp:880-920 */
  for (int i = 0; i < n; i++) {
    const double qi = s->coulomb_constant * s->charge[i];
    for (int j = i + 1; j < n; j++) {
      double d[3];
      for (int a = 0; a < 3; a++) d[a] = c[3 * j + a] - c[3 * i + a];
      const double r2 = dot3(d, d);
      const double qiqj = qi * s->charge[j];
      const double ij_born = rad[i] * rad[j];
      const double efac = exp(-r2 / (4.0 * ij_born));
      const double fgbi = 1.0 / sqrt(r2 + ij_born * efac);
      const double fgbk = -kappa * GB_KSCALE / fgbi;
      const double expmkf = exp(fgbk) / diel;
      const double dielfac = 1.0 - expmkf;
      egb -= qiqj * dielfac * fgbi;
      const double temp4 = fgbi * fgbi * fgbi;
      const double temp6 = qiqj * temp4 * (dielfac + fgbk * expmkf);
      const double fmag = temp6 * (1.0 - 0.25 * efac);
      const double temp5 = 0.5 * efac * temp6 * (ij_born + 0.25 * r2);
      sde[i] += rad[i] * temp5;
      sde[j] += rad[j] * temp5;
      if (f) {
        for (int a = 0; a < 3; a++) {
          f[3 * i + a] += fmag * d[a];
          f[3 * j + a] -= fmag * d[a];
        }
      }
    }
  }
  *e_gb += egb;

  /* Chain-rule prefactor for the OBC radii, nonbonded_potential.tpp:994-1021 */
  if (s->igb != ORC_GB_HCT) {
    for (int i = 0; i < n; i++) {
      const double rho = s->pb_radii[i] - offset;
      const double fipsi = psi[i] * (-rho);
      const double thi = tanh((s->gb_alpha[i] - (s->gb_beta[i] - s->gb_gamma[i] * fipsi) * fipsi) *
                              fipsi);
      sde[i] *= (s->gb_alpha[i] - (2.0 * s->gb_beta[i] - 3.0 * s->gb_gamma[i] * fipsi) * fipsi) *
                (1.0 - thi * thi) * rho / s->pb_radii[i];
    }
  }

  /* Pass 3: radius chain-rule forces, nonbonded_potential.tpp:1098-1244 */
  if (f) {
    for (int i = 0; i < n; i++) {
      const double rho_i = s->pb_radii[i] - offset;
      const double si = s->gb_screen[i] * rho_i;
      for (int j = i + 1; j < n; j++) {
        const double rho_j = s->pb_radii[j] - offset;
        const double sj = s->gb_screen[j] * rho_j;
        double d[3];
        for (int a = 0; a < 3; a++) d[a] = c[3 * j + a] - c[3 * i + a];
        const double r = sqrt(dot3(d, d));
        double fmag = hct_derivative(r, rho_i, sj) * sde[i] +
                      hct_derivative(r, rho_j, si) * sde[j];
        if (neck && r < rho_i + rho_j + 2.0 * offset + s->neck_cut) {
          /* nonbonded_potential.tpp:1219-1245 */
          double dij, dji;
          neck_term(s, i, j, r, nscale, &dij);
          neck_term(s, j, i, r, nscale, &dji);
          fmag += dij * sde[i] + dji * sde[j];
        }
        for (int a = 0; a < 3; a++) {
          f[3 * i + a] -= fmag * d[a];
          f[3 * j + a] += fmag * d[a];
        }
      }
    }
  }
  if (psi_out) memcpy(psi_out, psi, (size_t)n * sizeof(double));
  if (radii_out) memcpy(radii_out, rad, (size_t)n * sizeof(double));
  if (sdeijda_out) memcpy(sdeijda_out, sde, (size_t)n * sizeof(double));
  free(psi);
  free(rad);
  free(sde);
}

void orc_evaluate(const orc_system* s, const double* coords, double* forces, double* energies,
                  double* psi, double* radii, double* sumdeijda, int terms) {
  orc_evaluate_clash(s, coords, forces, energies, psi, radii, sumdeijda, terms, 0.0, 0.0);
}

void orc_evaluate_clash(const orc_system* s, const double* coords, double* forces,
                        double* energies, double* psi, double* radii, double* sumdeijda,
                        int terms, double clash_distance, double clash_ratio) {
  for (int t = 0; t < ORC_NTERMS; t++) energies[t] = 0.0;
  if (forces) memset(forces, 0, (size_t)s->natom * 3 * sizeof(double));
  if (terms & 1) {
    for (int t = 0; t < s->nbond; t++) {
      energies[ORC_BOND] += bond_term(coords, forces, s->bond_i[t], s->bond_j[t], s->bond_k[t],
                                      s->bond_r0[t]);
    }
    for (int t = 0; t < s->nangl; t++) {
      energies[ORC_ANGLE] += angle_term(coords, forces, s->angl_i[t], s->angl_j[t], s->angl_k[t],
                                        s->angl_keq[t], s->angl_theta0[t]);
    }
    for (int t = 0; t < s->ndihe; t++) {
      const double e = dihedral_term(coords, forces, s->dihe_i[t], s->dihe_j[t], s->dihe_k[t],
                                     s->dihe_l[t], s->dihe_amp[t], s->dihe_phase[t],
                                     s->dihe_freq[t]);
      energies[(s->dihe_improper && s->dihe_improper[t]) ? ORC_IMPROPER_DIHEDRAL :
                                                          ORC_PROPER_DIHEDRAL] += e;
      if (s->dihe_scee[t] > 0.0) {
        pair14_term(s, coords, forces, s->dihe_i[t], s->dihe_l[t], s->dihe_scee[t],
                    s->dihe_scnb[t], clash_distance, clash_ratio, &energies[ORC_ELEC_ONE_FOUR],
                    &energies[ORC_VDW_ONE_FOUR]);
      }
    }
  }
  if (terms & 2) {
    nonbonded_terms(s, coords, forces, clash_distance, clash_ratio, &energies[ORC_ELECTROSTATIC],
                    &energies[ORC_VDW]);
  }
  if ((terms & 4) && s->igb != ORC_GB_NONE) {
    gb_terms(s, coords, forces, &energies[ORC_GENERALIZED_BORN], psi, radii, sumdeijda);
  }
}

static double sq(double x) { return x * x; }

/* Root-sum-square of the contributions per term (test infrastructure: the scale of the rounding
 * error of a sum of independently rounded FP32 contributions).  Same loops as the evaluators
 * above; squares are summed here and square-rooted at the end. */
void orc_energy_magnitudes(const orc_system* s, const double* c, const double* radii,
                           double* mags) {
  for (int t = 0; t < ORC_NTERMS; t++) mags[t] = 0.0;
  const int n = s->natom;
  for (int t = 0; t < s->nbond; t++) {
    mags[ORC_BOND] += sq(bond_term(c, NULL, s->bond_i[t], s->bond_j[t], s->bond_k[t],
                                   s->bond_r0[t]));
  }
  for (int t = 0; t < s->nangl; t++) {
    mags[ORC_ANGLE] += sq(angle_term(c, NULL, s->angl_i[t], s->angl_j[t], s->angl_k[t],
                                     s->angl_keq[t], s->angl_theta0[t]));
  }
  for (int t = 0; t < s->ndihe; t++) {
    const double e = dihedral_term(c, NULL, s->dihe_i[t], s->dihe_j[t], s->dihe_k[t],
                                   s->dihe_l[t], s->dihe_amp[t], s->dihe_phase[t],
                                   s->dihe_freq[t]);
    mags[(s->dihe_improper && s->dihe_improper[t]) ? ORC_IMPROPER_DIHEDRAL :
                                                    ORC_PROPER_DIHEDRAL] += sq(e);
    if (s->dihe_scee[t] > 0.0) {
      const int i = s->dihe_i[t], l = s->dihe_l[t];
      double d[3];
      for (int a = 0; a < 3; a++) d[a] = c[3 * l + a] - c[3 * i + a];
      const double invr2 = 1.0 / dot3(d, d);
      const double invr6 = invr2 * invr2 * invr2;
      const int ty = s->lj_idx[i] * s->n_lj_types + s->lj_idx[l];
      mags[ORC_ELEC_ONE_FOUR] += sq(s->coulomb_constant * s->charge[i] * s->charge[l] /
                                    s->dihe_scee[t] * sqrt(invr2));
      mags[ORC_VDW_ONE_FOUR] += sq((fabs(s->lja14[ty]) * invr6 + fabs(s->ljb14[ty])) * invr6 /
                                   s->dihe_scnb[t]);
    }
  }
  char* excl = (char*)calloc((size_t)n, 1);
  for (int i = 0; i < n; i++) {
    for (int e = s->excl_bounds[i]; e < s->excl_bounds[i + 1]; e++) excl[s->excl_list[e]] = 1;
    for (int j = i + 1; j < n; j++) {
      if (excl[j]) continue;
      double d[3];
      for (int a = 0; a < 3; a++) d[a] = c[3 * j + a] - c[3 * i + a];
      const double invr2 = 1.0 / dot3(d, d);
      const double invr6 = invr2 * invr2 * invr2;
      const int ty = s->lj_idx[j] * s->n_lj_types + s->lj_idx[i];
      mags[ORC_ELECTROSTATIC] += sq(s->coulomb_constant * s->charge[i] * s->charge[j] *
                                    sqrt(invr2));
      mags[ORC_VDW] += sq((fabs(s->lja[ty]) * invr6 + fabs(s->ljb[ty])) * invr6);
    }
    for (int e = s->excl_bounds[i]; e < s->excl_bounds[i + 1]; e++) excl[s->excl_list[e]] = 0;
  }
  free(excl);
  if (s->igb != ORC_GB_NONE && radii) {
    const double kappa = (s->saltcon > 1.0e-8) ? sqrt(GB_SALT_KAPPA * s->saltcon) : 0.0;
    for (int i = 0; i < n; i++) {
      const double expmkf = exp(-GB_KSCALE * kappa * radii[i]) / s->dielectric;
      mags[ORC_GENERALIZED_BORN] += sq(0.5 * s->charge[i] * s->charge[i] *
                                       s->coulomb_constant * (1.0 - expmkf) / radii[i]);
      for (int j = i + 1; j < n; j++) {
        double d[3];
        for (int a = 0; a < 3; a++) d[a] = c[3 * j + a] - c[3 * i + a];
        const double r2 = dot3(d, d);
        const double ijb = radii[i] * radii[j];
        const double fgbi = 1.0 / sqrt(r2 + ijb * exp(-r2 / (4.0 * ijb)));
        const double expm = exp(-kappa * GB_KSCALE / fgbi) / s->dielectric;
        mags[ORC_GENERALIZED_BORN] += sq(s->coulomb_constant * s->charge[i] * s->charge[j] *
                                         (1.0 - expm) * fgbi);
      }
    }
  }
  for (int t = 0; t < ORC_NTERMS; t++) mags[t] = sqrt(mags[t]);
}

/* ---------------------------------------------------------------------------------------------
 * Line minimization following the batched GPU driver
 * ------------------------------------------------------------------------------------------- */
static double total_energy(const double* e) {
  double s = 0.0;
  for (int t = 0; t < ORC_NTERMS; t++) s += e[t];
  return s;
}

/* Solve the 4x4 system for the cubic through (x_k, e_k), Gauss-Jordan with partial pivoting
 * (line_movement.cui:160-236 performs the same elimination) */
static void cubic_fit(const double* x, const double* e, double* abcd) {
  double m[4][5];
  for (int r = 0; r < 4; r++) {
    m[r][0] = x[r] * x[r] * x[r];
    m[r][1] = x[r] * x[r];
    m[r][2] = x[r];
    m[r][3] = 1.0;
    m[r][4] = e[r];
  }
  for (int col = 0; col < 4; col++) {
    int piv = col;
    for (int r = col + 1; r < 4; r++) {
      if (fabs(m[r][col]) > fabs(m[piv][col])) piv = r;
    }
    if (piv != col) {
      for (int k = 0; k < 5; k++) {
        const double t = m[col][k];
        m[col][k] = m[piv][k];
        m[piv][k] = t;
      }
    }
    const double p = m[col][col];
    for (int k = 0; k < 5; k++) m[col][k] /= p;
    for (int r = 0; r < 4; r++) {
      if (r == col) continue;
      const double fac = m[r][col];
      for (int k = 0; k < 5; k++) m[r][k] -= fac * m[col][k];
    }
  }
  for (int r = 0; r < 4; r++) abcd[r] = m[r][4];
}

void orc_minimize(const orc_system* s, double* coords, int maxcyc, int sd_cycles, double dx0,
                  double* history) {
  orc_minimize_ex(s, coords, maxcyc, sd_cycles, dx0, 0.0, history, NULL);
}

void orc_minimize_ex(const orc_system* s, double* coords, int maxcyc, int sd_cycles, double dx0,
                     double drms, double* history, int* cycles_run) {
  orc_minimize_clash(s, coords, maxcyc, sd_cycles, dx0, drms, 0, 0.0, 0.0, history, cycles_run);
}

void orc_minimize_clash(const orc_system* s, double* coords, int maxcyc, int sd_cycles,
                        double dx0, double drms, int clash_cycles, double clash_distance,
                        double clash_ratio, double* history, int* cycles_run) {
  const int n = s->natom;
  const size_t nb = (size_t)n * 3 * sizeof(double);
  double* frc = (double*)malloc(nb);
  double* prv = (double*)calloc((size_t)n * 3, sizeof(double));
  double* cgt = (double*)calloc((size_t)n * 3, sizeof(double));
  double* dir = (double*)malloc(nb);
  double e[ORC_NTERMS];
  double l_move = dx0;
  int done_at = maxcyc;
  for (int cyc = 0; cyc < maxcyc; cyc++) {
    /* clash damping for the first clash_cycles cycles, the softened cores shrinking linearly
     * (minimization.tpp:224-228, hpc_minimization.cu:268-272) */
    double cd = 0.0, cr = 0.0;
    if (cyc < clash_cycles) {
      const double progress = (double)(clash_cycles - cyc) / (double)clash_cycles;
      cd = clash_distance * progress;
      cr = clash_ratio * progress;
    }
    /* force + energy evaluation at the start of the cycle */
    orc_evaluate_clash(s, coords, frc, e, NULL, NULL, NULL, 7, cd, cr);
    const double e0 = total_energy(e);
    if (history) history[cyc] = e0;
    if (drms > 0.0) {
      double ff = 0.0;
      for (int k = 0; k < 3 * n; k++) ff += frc[k] * frc[k];
      if (sqrt(ff / (3.0 * n)) <= drms) {
        done_at = cyc;
        break;
      }
    }

    /* conjugate gradient direction, Math/conjugate_gradient.cui:8-140 and
     * hpc_reduction.cu:154-300; the step counter has been advanced once before this call
     * (hpc_minimization.cu:470) */
    double gg = 0.0, dgg = 0.0;
    for (int k = 0; k < 3 * n; k++) {
      gg += prv[k] * prv[k];
      dgg += (frc[k] - prv[k]) * frc[k];
    }
    const int step = cyc + 1;
    double gam = (step >= sd_cycles && gg > 0.0) ? dgg / gg : 0.0;
    double msum = 0.0;
    for (int k = 0; k < 3 * n; k++) {
      prv[k] = frc[k];
      if (fabs(gam) > VERYTINY) {
        cgt[k] = frc[k] + gam * cgt[k];
      }
      else {
        cgt[k] = frc[k];
      }
      msum += cgt[k] * cgt[k];
    }
    const double inv_norm = (msum > 0.0) ? 1.0 / sqrt(msum) : 0.0;
    for (int k = 0; k < 3 * n; k++) dir[k] = cgt[k] * inv_norm;

    /* three trial moves along the line, line_movement.cui:88-126 */
    const double s_move = l_move;
    double ev[4], mv[4];
    ev[0] = e0;
    mv[0] = 0.0;
    double mfac = 1.0;
    double cum = 0.0;
    for (int mvn = 0; mvn < 3; mvn++) {
      if (mvn == 1) {
        mfac = (ev[1] < ev[0]) ? 1.04 : 0.8;
      }
      else if (mvn == 2) {
        mfac = mfac * ((ev[2] < ev[1]) ? 1.03 : 0.85);
      }
      for (int k = 0; k < 3 * n; k++) coords[k] += dir[k] * mfac * s_move;
      cum += mfac;
      mv[mvn + 1] = cum;
      orc_evaluate_clash(s, coords, NULL, e, NULL, NULL, NULL, 7, cd, cr);
      ev[mvn + 1] = total_energy(e);
    }

    /* cubic fit and final placement, line_movement.cui:236-330 */
    double move_factor, new_base;
    if (ev[0] < ev[1] && ev[0] < ev[2] && ev[0] < ev[3]) {
      move_factor = -mv[3];
      new_base = 0.8;
    }
    else {
      double abcd[4];
      cubic_fit(mv, ev, abcd);
      const double d0 = 3.0 * abcd[0], d1 = 2.0 * abcd[1], d2 = abcd[2];
      const double sqrt_arg = d1 * d1 - 4.0 * d0 * d2;
      if (sqrt_arg < 0.0) {
        if (ev[0] < ev[3]) {
          move_factor = -mv[3];
          new_base = 0.8;
        }
        else {
          move_factor = 0.0;
          new_base = 1.2;
        }
      }
      else {
        const double ext_i = (-d1 + sqrt(sqrt_arg)) / (2.0 * d0);
        const double ext_ii = (-d1 - sqrt(sqrt_arg)) / (2.0 * d0);
        const double min_pos = (2.0 * d0 * ext_i + d1 > 0.0) ? ext_i : ext_ii;
        if (min_pos <= 0.0) {
          if (ev[3] >= ev[0]) {
            move_factor = -mv[3];
            new_base = 0.8;
          }
          else {
            move_factor = 0.0;
            new_base = 1.2;
          }
        }
        else if (min_pos < mv[3]) {
          const double epred = ((abcd[0] * min_pos + abcd[1]) * min_pos + abcd[2]) * min_pos +
                               abcd[3];
          if (epred > ev[0]) {
            move_factor = -mv[3];
            new_base = 0.8;
          }
          else if (epred < ev[3]) {
            move_factor = min_pos - mv[3];
            new_base = (min_pos > 0.6) ? 1.05 : 0.95;
          }
          else {
            move_factor = 0.0;
            new_base = 1.05;
          }
        }
        else {
          move_factor = 0.0;
          new_base = 1.05;
        }
      }
    }
    l_move = s_move * new_base;
    if (fabs(move_factor) > VERYTINY) {
      for (int k = 0; k < 3 * n; k++) coords[k] += dir[k] * move_factor * s_move;
    }
  }
  orc_evaluate(s, coords, NULL, e, NULL, NULL, NULL, 7);
  if (history) history[done_at] = total_energy(e);
  if (cycles_run) *cycles_run = done_at;
  free(frc);
  free(prv);
  free(cgt);
  free(dir);
}

/* ---------------------------------------------------------------------------------------------
 * Split fixed-point conversions, Numerics/accumulation.cui:126-160
 * ------------------------------------------------------------------------------------------- */
void orc_float_to_int63(float v, int32_t* x, int32_t* y) {
  const float lim = 2147483648.0f;
  if (fabsf(v) >= lim) {
    const int spill = (int)(v / lim);
    *x = (int32_t)rintf(v - (float)spill * lim);
    *y = spill;
  }
  else {
    *x = (int32_t)rintf(v);
    *y = 0;
  }
}

void orc_double_to_int95(double v, int64_t* x, int32_t* y) {
  const double lim = 9223372036854775808.0;
  if (fabs(v) >= lim) {
    const int spill = (int)(v / lim);
    *x = (int64_t)llrint(v - (double)spill * lim);
    *y = spill;
  }
  else {
    *x = (int64_t)llrint(v);
    *y = 0;
  }
}
