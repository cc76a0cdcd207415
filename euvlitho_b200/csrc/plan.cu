// Plans: the configuration tables of the reference drivers, built on the host
// in C++, and run functions that chain the library's entry points the way
// intensity.cpp main (Abbe image), m3d.cpp main (M3D parameters) and ampS over
// the NA-circle sources do.  With these a C or C++ caller needs no other host
// code: euv_plan_create -> euv_plan_upload -> euv_plan_intensity / _m3d.
//
// Table builders (each follows the reference loop it names):
//   order_set      intensity.cpp:148-164 (rounded diamond), m3d.cpp:113-129
//                  (ellipse), or an explicit box; l outer, m inner
//   pupil_set      intensity.cpp:166-195, m3d.cpp:160-195 (xinput = snum >= 8)
//   sources        source(), intensity.cpp:467-502
//   rotate         intensity.cpp:423-465
//   abbe_table     intensity.cpp:248-353 (E = i k R A / sqrt(k^2 - k_s^2),
//                  pupil phase with z0 and defocus)
//   na_sources     header.h:1394-1397
// Device memory is the caller's: the tables go into a caller buffer
// (euv_plan_upload), every run takes a caller workspace.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace euv {
namespace {

const double kPi = std::atan(1.0) * 4.0;  // intensity.cpp:55

struct Fam {
  int nsx, nsy;
  std::vector<std::pair<int, int>> pts;
};

// Byte layout of the device tables (offsets from the caller's base).
struct DevLayout {
  size_t lidx, midx;                                  // [N]
  size_t u_kx0, u_ky0, u_pol, u_clip, u_order, u_kz2;  // per unit, max_clips * ntab
  size_t u_tab, u_img, u_nsrc, inv_w;                 // Abbe per unit / per image
  size_t coef, nidx, px, py, row_start;               // Abbe tables
  size_t na_l, na_m, na_order;                        // NA sources (wide order index)
  size_t n_lidx, n_midx, n_kx0, n_ky0, n_pol, n_spec, n_order, n_kz2;  // narrow solves
  size_t src_nn, lin, min_, xin, pair;                // M3D fit tables
  size_t ax_vc, ax_ab;                                // narrow-solve results
  size_t status;
  size_t total;
};

struct Carve {
  size_t off = 0;
  template <typename T>
  size_t take(size_t count) {
    const size_t o = off;
    off += ((count * sizeof(T)) + 255) & ~(size_t)255;
    return o;
  }
};

}  // namespace
}  // namespace euv

struct euv_plan {
  euv_config cfg;
  euv_plan_info info;
  // host tables
  std::vector<int> lidx, midx;
  std::map<std::pair<int, int>, int> pos;
  std::vector<int> lin, min_, xin, snum;
  std::vector<euv::Fam> fams;
  std::vector<int> na_l, na_m, na_order;
  int ntab = 0, n_src = 0;
  std::vector<double> tab_kx0, tab_ky0;
  std::vector<int> tab_pol, tab_nsrc;
  std::vector<int> tab_order;    // [ntab][n_src]
  std::vector<double> tab_kz2;   // [ntab][n_src]
  std::vector<euv_c64> coef;     // [ntab][n_src][ncut][3]
  std::vector<int> nidx;         // [ntab][n_src][ncut]
  std::vector<int> row_start;
  // M3D
  std::string m3d_error;         // empty when the M3D tables exist
  int lmax_n = 0, mmax_n = 0;
  std::vector<int> nlidx, nmidx, src_nn, pair;
  int s_center = -1;
  // device
  int max_clips = 0;
  char* dev = nullptr;
  euv::DevLayout L{};
  std::vector<char> staging;
  bool uniform_done = false;
};

namespace euv {
namespace {

struct Cfg {
  const euv_config& c;
  double dx() const { return (double)c.ndivx; }
  double dy() const { return (double)c.ndivy; }
  double k() const { return 2.0 * kPi / c.wavelength; }
  int fdivx() const { return (int)(dx() / c.delta + 0.000001); }
  int fdivy() const { return (int)(dy() / c.delta + 0.000001); }
  double kx0() const {
    const double phi0 = 90.0 - c.azimuth;
    return k() * std::sin(kPi / 180.0 * c.theta0) * std::cos(kPi / 180.0 * phi0);
  }
  double ky0() const {
    const double phi0 = 90.0 - c.azimuth;
    return k() * std::sin(kPi / 180.0 * c.theta0) * std::sin(kPi / 180.0 * phi0);
  }
  double z0() const {
    double s = 0.0;
    for (int n = 0; n < c.n_slices; ++n) s += c.dabs[n];
    return s + c.z0_offset;
  }
  int lsx() const { return (int)(c.na * dx() / (double)c.mx / c.wavelength + 1); }
  int lsy() const { return (int)(c.na * dy() / (double)c.my / c.wavelength + 1); }
  int lpx() const { return (int)(c.na * dx() / (double)c.mx * 2 / c.wavelength + 0.0001); }
  int lpy() const { return (int)(c.na * dy() / (double)c.my * 2 / c.wavelength + 0.0001); }
  int ndivs() const {
    if (c.ndivs > 0) return c.ndivs;
    const int n = (int)(180.0 / kPi * c.wavelength / dx() / c.sigmadiv);
    return n < 1 ? 1 : n;
  }
  // order_limits of the drivers (intensity.cpp:139-146, m3d.cpp:101-111)
  void limits(int kind, double cut, int* L, int* M) const {
    if (kind == EUV_ORDERS_BOX) {
      *L = c.lbox;
      *M = c.mbox;
      return;
    }
    const double cutx = c.na / (double)c.mx * cut, cuty = c.na / (double)c.my * cut;
    *L = (int)(cutx * dx() / c.wavelength);
    *M = (int)(cuty * dy() / c.wavelength);
  }
  bool in_na(double l, double m) const {
    const double a = (l * c.mx) / dx(), b = (m * c.my) / dy(), r = c.na / c.wavelength;
    return a * a + b * b <= r * r;
  }
};

void order_set(int kind, int L, int M, std::vector<int>& li, std::vector<int>& mi) {
  li.clear();
  mi.clear();
  for (int l = -L; l <= L; ++l)
    for (int m = -M; m <= M; ++m) {
      bool keep = true;
      if (kind == EUV_ORDERS_DIAMOND) {
        keep = (std::abs(l) / (double)(L + 0.01) + 1.0) * (std::abs(m) / (double)(M + 0.01) + 1.0) <=
               2.0;
      } else if (kind == EUV_ORDERS_ELLIPSE) {
        const double a = l / (double)(L + 0.01), b = m / (double)(M + 0.01);
        keep = a * a + b * b <= 1.0;
      }
      if (keep) {
        li.push_back(l);
        mi.push_back(m);
      }
    }
}

struct V3 {
  double x, y, z;
};
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 unit(V3 a) {
  const double n = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return {a.x / n, a.y / n, a.z / n};
}
V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }

// R (3x2, row-major R[i][j]) of rotate(), intensity.cpp:423-465
void rotate(double k, int MX, int MY, double px, double py, double sx0, double sy0, double R[3][2]) {
  const V3 s0{sx0, sy0, -std::sqrt(k * k - sx0 * sx0 - sy0 * sy0)};
  const V3 p{px, py, 0.0};
  const V3 pp{MX * px, MY * py, -std::sqrt(k * k - MX * px * MX * px - MY * py * MY * py)};
  const V3 ez{0.0, 0.0, 1.0};
  V3 es, esp, em, emp;
  if (px * px + py * py > 0.00001) {
    es = unit(cross(p, s0));
    esp = unit(cross(pp, ez));
    em = cross(es, unit(V3{p.x + s0.x, p.y + s0.y, p.z + s0.z}));
    emp = scale(cross(esp, pp), 1.0 / k);
  } else {
    es = unit(cross(ez, s0));
    esp = scale(es, -1.0);
    em = scale(cross(es, s0), 1.0 / k);
    emp = cross(esp, V3{0.0, 0.0, -1.0});
  }
  const double e[3] = {esp.x, esp.y, esp.z}, m[3] = {emp.x, emp.y, emp.z};
  const double s[2] = {es.x, es.y}, t[2] = {em.x, em.y};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 2; ++j) R[i][j] = e[i] * s[j] + m[i] * t[j];
}

int fail(const char* msg) {
  euv_set_error("euv_plan: %s", msg);
  return EUV_ERR_BAD_ARG;
}

int build(euv_plan* P) {
  const euv_config& c = P->cfg;
  const Cfg g{c};
  if (c.ndivx <= 0 || c.ndivy <= 0 || c.delta <= 0 || c.wavelength <= 0 || c.na <= 0 ||
      c.mx <= 0 || c.my <= 0 || c.n_slices < 1 || c.n_slices > EUV_MAX_SLICES ||
      c.illum_type < 0 || c.illum_type > 3 || c.n_pols < 1 || c.n_pols > 2 ||
      (c.precision != EUV_PREC_FP64 && c.precision != EUV_PREC_MIXED) ||
      c.order_kind < EUV_ORDERS_DIAMOND || c.order_kind > EUV_ORDERS_BOX || c.sigmadiv <= 0)
    return fail("invalid configuration field");
  for (int p = 0; p < c.n_pols; ++p)
    if (c.pols[p] != 0 && c.pols[p] != 1) return fail("polarisation must be 0 (X) or 1 (Y)");
  if (c.n_pols == 2 && c.pols[0] == c.pols[1]) return fail("the two polarisations must differ");
  if (g.fdivx() % c.ndivx || g.fdivy() % c.ndivy)
    return fail("the Fourier grid must refine the mask grid by an integer factor");
  if (c.ndivx % c.mx || c.ndivy % c.my) return fail("the clip must be a multiple of MX, MY pixels");
  const double k = g.k(), dx = g.dx(), dy = g.dy(), kx0 = g.kx0(), ky0 = g.ky0();
  const int MX = c.mx, MY = c.my;
  const double NA = c.na;
  int L, M;
  g.limits(c.order_kind, c.cut, &L, &M);
  if (L < 0 || M < 0) return fail("negative order limits");
  order_set(c.order_kind, L, M, P->lidx, P->midx);
  const int N = (int)P->lidx.size();
  if (N == 0) return fail("empty order set");
  for (int i = 0; i < N; ++i) P->pos[{P->lidx[i], P->midx[i]}] = i;
  {
    const double ax = std::fabs(kx0) + 2 * kPi * (L + 1) / dx;
    const double ay = std::fabs(ky0) + 2 * kPi * (M + 1) / dy;
    if (ax * ax + ay * ay >= k * k)
      return fail("order set reaches evanescent orders (|k_xy| >= k); the reference computes NaN "
                  "for them (header.h:1283); reduce the order cut");
  }
  // pupil set (l-major) with snum and xinput
  const int lsx = g.lsx(), lsy = g.lsy(), lpx = g.lpx(), lpy = g.lpy();
  for (int lp = -lpx; lp <= lpx; ++lp)
    for (int mp = -lpy; mp <= lpy; ++mp) {
      int sn = 0;
      for (int ls = -lsx; ls <= lsx; ++ls)
        for (int ms = -lsy; ms <= lsy; ++ms)
          if (g.in_na(ls, ms) && g.in_na(lp + ls, mp + ms)) ++sn;
      if (sn > 0) {
        P->lin.push_back(lp);
        P->min_.push_back(mp);
        P->snum.push_back(sn);
        P->xin.push_back(sn >= 8 ? 1 : 0);
      }
    }
  const int ncut = (int)P->lin.size();
  if (ncut == 0) return fail("empty pupil set");
  // source families (source(), intensity.cpp:467-502)
  const int ndivs = g.ndivs();
  {
    const double dkx = 2.0 * kPi / dx, dky = 2.0 * kPi / dy;
    const int l0max = (int)(k * NA / MX * c.sigma1 / dkx + 1);
    const int m0max = (int)(k * NA / MY * c.sigma1 / dky + 1);
    const double tan_half = std::tan(kPi * c.openangle / 180.0 / 2.0);
    const double s1 = c.sigma1, s2 = c.sigma2;
    const int t = c.illum_type;
    int total = 0;
    for (int nsx = 0; nsx < ndivs; ++nsx)
      for (int nsy = 0; nsy < ndivs; ++nsy) {
        Fam f{nsx, nsy, {}};
        for (int l = -l0max; l <= l0max; ++l)
          for (int m = -m0max; m <= m0max; ++m) {
            const double skx = l * dkx + 2.0 * kPi / dx * nsx / (double)ndivs;
            const double sky = m * dky + 2.0 * kPi / dy * nsy / (double)ndivs;
            const double skxo = skx * MX, skyo = sky * MY;
            const double r2 = skxo * skxo + skyo * skyo;
            const double r = std::sqrt(r2);
            const double R1 = k * NA * s1, R2 = k * NA * s2;
            const bool ring = r <= R1 && r >= R2;
            const bool ok = (t == 0 && r2 <= R1 * R1) || (t == 1 && ring) ||
                            (t == 2 && ring && std::fabs(skyo) <= std::fabs(skxo) * tan_half) ||
                            (t == 3 && ring && std::fabs(skxo) <= std::fabs(skyo) * tan_half);
            if (ok && (c.max_sources <= 0 || total < c.max_sources)) {
              f.pts.push_back({l, m});
              ++total;
            }
          }
        if (!f.pts.empty()) P->fams.push_back(f);
      }
    if (total == 0) return fail("the illumination has no source point");
  }
  const int nf = (int)P->fams.size();
  int nsmax = 0, sdivsum = 0;
  for (const Fam& f : P->fams) {
    nsmax = std::max(nsmax, (int)f.pts.size());
    sdivsum += (int)f.pts.size();
  }
  P->n_src = nsmax;
  P->ntab = c.n_pols * nf;
  // Abbe tables per (polarisation, family) and the source columns of ampS
  const double z0 = g.z0(), z = c.z;
  P->coef.assign((size_t)P->ntab * nsmax * ncut * 3, euv_c64{0.0, 0.0});
  P->nidx.assign((size_t)P->ntab * nsmax * ncut, -1);
  P->tab_order.assign((size_t)P->ntab * nsmax, -1);
  P->tab_kz2.assign((size_t)P->ntab * nsmax, 0.0);
  for (int pi = 0; pi < c.n_pols; ++pi)
    for (int fi = 0; fi < nf; ++fi) {
      const Fam& f = P->fams[fi];
      const int t = pi * nf + fi;
      const double sx0 = 2.0 * kPi / dx * f.nsx / (double)ndivs + kx0;
      const double sy0 = 2.0 * kPi / dy * f.nsy / (double)ndivs + ky0;
      P->tab_kx0.push_back(sx0);
      P->tab_ky0.push_back(sy0);
      P->tab_pol.push_back(c.pols[pi]);
      P->tab_nsrc.push_back((int)f.pts.size());
      for (int s = 0; s < (int)f.pts.size(); ++s) {
        const int l0 = f.pts[s].first, m0 = f.pts[s].second;
        // source column of ampS (header.h:1396-1409)
        const double kxs = sx0 + l0 * 2.0 * kPi / dx, kys = sy0 + m0 * 2.0 * kPi / dy;
        auto it = P->pos.find({l0, m0});
        if (it == P->pos.end()) return fail("a source order of a family is outside the order set");
        P->tab_order[(size_t)t * nsmax + s] = it->second;
        P->tab_kz2[(size_t)t * nsmax + s] = 2.0 * std::sqrt(k * k - kxs * kxs - kys * kys);
        // E-field factors (intensity.cpp:276-353)
        const double kx = sx0 + 2.0 * kPi / dx * l0, ky = sy0 + 2.0 * kPi / dy * m0;
        for (int i = 0; i < ncut; ++i) {
          const double kxn = 2.0 * kPi / dx * f.nsx / (double)ndivs + 2.0 * kPi / dx * l0 +
                             2.0 * kPi * P->lin[i] / dx;
          const double kyn = 2.0 * kPi / dy * f.nsy / (double)ndivs + 2.0 * kPi / dy * m0 +
                             2.0 * kPi * P->min_[i] / dy;
          if (!(MX * MX * kxn * kxn + MY * MY * kyn * kyn <= (NA * k) * (NA * k))) continue;
          auto o = P->pos.find({l0 + P->lin[i], m0 + P->min_[i]});
          if (o == P->pos.end())
            return fail("the order set misses a pupil order of a source (the reference reads "
                        "its -1000 sentinel there, intensity.cpp:297-299); widen the order set");
          double R[3][2];
          rotate(k, MX, MY, kxn, kyn, kx0, ky0, R);
          const double ph = ((kxn + kx0) * (kxn + kx0) + (kyn + ky0) * (kyn + ky0)) / 2.0 / k * z0 +
                            (MX * MX * kxn * kxn + MY * MY * kyn * kyn) / 2.0 / k * z;
          const double cr = std::cos(ph), ci = std::sin(ph);
          const int col = c.pols[pi];  // X: R(:,0), Y: R(:,1)
          const double den = col == 0 ? std::sqrt(k * k - kx * kx) : std::sqrt(k * k - ky * ky);
          const size_t e = ((size_t)t * nsmax + s) * ncut + i;
          P->nidx[e] = o->second;
          for (int q = 0; q < 3; ++q) {
            // f = i k R(q, col) / den, times exp(i ph)
            const double fi_ = k * R[q][col] / den;  // f = (0, fi_)
            P->coef[e * 3 + q] = euv_c64{-fi_ * ci, fi_ * cr};
          }
        }
      }
    }
  // row_start[j] = first pupil point with lin >= j - lpx, j in [0, 2 lpx + 1]
  for (int j = 0; j <= 2 * lpx + 1; ++j) {
    int r = 0;
    while (r < ncut && P->lin[r] < j - lpx) ++r;
    P->row_start.push_back(r);
  }
  // NA-circle sources of ampS (header.h:1394-1397) and the M3D tables
  for (int ls = -lsx; ls <= lsx; ++ls)
    for (int ms = -lsy; ms <= lsy; ++ms)
      if (g.in_na(ls, ms)) {
        P->na_l.push_back(ls);
        P->na_m.push_back(ms);
        auto it = P->pos.find({ls, ms});
        P->na_order.push_back(it == P->pos.end() ? -1 : it->second);
      }
  const int nna = (int)P->na_l.size();
  for (int s = 0; s < nna; ++s)
    if (P->na_l[s] == 0 && P->na_m[s] == 0) P->s_center = s;
  for (int s = 0; s < nna; ++s)
    if (P->na_order[s] < 0) P->m3d_error = "the order set misses an NA-circle source order";
  g.limits(EUV_ORDERS_ELLIPSE, 1.5, &P->lmax_n, &P->mmax_n);  // m3d.cpp:107-129
  order_set(EUV_ORDERS_ELLIPSE, P->lmax_n, P->mmax_n, P->nlidx, P->nmidx);
  {
    std::map<std::pair<int, int>, int> npos;
    for (int i = 0; i < (int)P->nlidx.size(); ++i) npos[{P->nlidx[i], P->nmidx[i]}] = i;
    for (int s = 0; s < nna; ++s) {
      auto it = npos.find({P->na_l[s], P->na_m[s]});
      P->src_nn.push_back(it == npos.end() ? -1 : it->second);
      if (it == npos.end()) P->m3d_error = "the narrow order set misses a source order";
    }
  }
  if (P->s_center < 0) P->m3d_error = "no (0,0) source order";
  P->pair.assign((size_t)ncut * nna, -1);
  for (int n = 0; n < ncut && P->m3d_error.empty(); ++n)
    for (int s = 0; s < nna; ++s) {
      const int l = P->na_l[s] + P->lin[n], m = P->na_m[s] + P->min_[n];
      if (!g.in_na(l, m)) continue;
      auto it = P->pos.find({l, m});
      if (it == P->pos.end()) {
        P->m3d_error = "the order set misses a pupil order of the M3D fit";
        break;
      }
      P->pair[(size_t)n * nna + s] = it->second;
    }

  euv_plan_info& I = P->info;
  I.n_orders = N;
  I.lmax = L;
  I.mmax = M;
  I.ncut = ncut;
  I.lpx = lpx;
  I.lpy = lpy;
  I.lsx = lsx;
  I.lsy = lsy;
  I.n_na_sources = nna;
  I.ndivs = ndivs;
  I.n_families = nf;
  I.n_src_max = nsmax;
  I.sdivsum = sdivsum;
  I.n_pols = c.n_pols;
  I.units_per_clip = P->ntab;
  I.xdiv = c.ndivx / MX;
  I.ydiv = c.ndivy / MY;
  I.fdivx = g.fdivx();
  I.fdivy = g.fdivy();
  I.n_orders_narrow = (int)P->nlidx.size();
  I.k = k;
  I.kx0 = kx0;
  I.ky0 = ky0;
  I.z0 = z0;
  return EUV_OK;
}

DevLayout layout(const euv_plan* P, int max_clips) {
  const euv_plan_info& I = P->info;
  const size_t N = I.n_orders, U = (size_t)max_clips * P->ntab, ns = P->n_src;
  const size_t nna = I.n_na_sources, Nn = I.n_orders_narrow, ncut = I.ncut;
  Carve cv;
  DevLayout d{};
  d.lidx = cv.take<int>(N);
  d.midx = cv.take<int>(N);
  d.u_kx0 = cv.take<double>(U);
  d.u_ky0 = cv.take<double>(U);
  d.u_pol = cv.take<int>(U);
  d.u_clip = cv.take<int>(U);
  d.u_order = cv.take<int>(U * ns);
  d.u_kz2 = cv.take<double>(U * ns);
  d.u_tab = cv.take<int>(U);
  d.u_img = cv.take<int>(U);
  d.u_nsrc = cv.take<int>(U);
  d.inv_w = cv.take<double>((size_t)max_clips * I.n_pols);
  d.coef = cv.take<euv_c64>((size_t)P->ntab * ns * ncut * 3);
  d.nidx = cv.take<int>((size_t)P->ntab * ns * ncut);
  d.px = cv.take<int>(ncut);
  d.py = cv.take<int>(ncut);
  d.row_start = cv.take<int>(2 * (size_t)I.lpx + 2);
  d.na_l = cv.take<int>(nna);
  d.na_m = cv.take<int>(nna);
  d.na_order = cv.take<int>(nna);
  d.n_lidx = cv.take<int>(Nn);
  d.n_midx = cv.take<int>(Nn);
  d.n_kx0 = cv.take<double>(2);
  d.n_ky0 = cv.take<double>(2);
  d.n_pol = cv.take<int>(2);
  d.n_spec = cv.take<int>(2);
  d.n_order = cv.take<int>(2 * nna);
  d.n_kz2 = cv.take<double>(2 * nna);
  d.src_nn = cv.take<int>(nna);
  d.lin = cv.take<int>(ncut);
  d.min_ = cv.take<int>(ncut);
  d.xin = cv.take<int>(ncut);
  d.pair = cv.take<int>(ncut * nna);
  d.ax_vc = cv.take<euv_c64>(2 * nna * Nn);  // one ampS of two units: vacuum, then absorber
  d.ax_ab = d.ax_vc + nna * Nn * sizeof(euv_c64);
  d.status = cv.take<int>(1);
  d.total = cv.off;
  return d;
}

template <typename T>
void put(std::vector<char>& st, size_t off, const T* src, size_t n) {
  if (n) std::memcpy(st.data() + off, src, n * sizeof(T));
}

// Per-unit arrays of an ampS call at one incidence for the NA-circle sources:
// unit u = clip u, source columns = the NA sources (header.h:1396-1409).
__global__ void plan_na_units_kernel(int n_clips, int nna, double kx0, double ky0, int polar,
                                     double k, double dx, double dy, const int* na_l,
                                     const int* na_m, const int* na_order, double* u_kx0,
                                     double* u_ky0, int* u_pol, int* u_clip, int* u_order,
                                     double* u_kz2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_clips * nna) return;
  const int c = t / nna, s = t % nna;
  const double twopi = 6.283185307179586476925286766559;
  if (s == 0) {
    u_kx0[c] = kx0;
    u_ky0[c] = ky0;
    u_pol[c] = polar;
    u_clip[c] = c;
  }
  const double kx = kx0 + na_l[s] * twopi / dx, ky = ky0 + na_m[s] * twopi / dy;
  u_order[t] = na_order[s];
  u_kz2[t] = 2.0 * sqrt(k * k - kx * kx - ky * ky);
}

euv_amp_desc amp_base(const euv_plan* P) {
  const euv_config& c = P->cfg;
  euv_amp_desc d;
  std::memset(&d, 0, sizeof(d));
  d.n_orders = P->info.n_orders;
  d.lmax = P->info.lmax;
  d.mmax = P->info.mmax;
  d.d_lindex = reinterpret_cast<const int*>(P->dev + P->L.lidx);
  d.d_mindex = reinterpret_cast<const int*>(P->dev + P->L.midx);
  d.dx = (double)c.ndivx;
  d.dy = (double)c.ndivy;
  d.k = P->info.k;
  d.n_slices = c.n_slices;
  for (int n = 0; n < c.n_slices; ++n) {
    d.eabs[n] = c.eabs[n];
    d.dabs[n] = c.dabs[n];
  }
  d.refresh_sigma = c.refresh_sigma;
  d.stack = c.stack;
  d.precision = c.precision;
  d.m_max = 0;
  d.d_status = reinterpret_cast<int*>(P->dev + P->L.status);
  return d;
}

// Workspace size of an ampS descriptor whose per-unit pointers are not set yet:
// the query validates the descriptor (non-null pointers) but reads none of them.
size_t amp_bytes(euv_amp_desc d) {
  static const double dd = 0.0;
  static const int di = 0;
  d.d_kx0 = d.d_ky0 = d.d_src_2kz = &dd;
  d.d_polar = d.d_spec = d.d_src_order = &di;
  if (!d.d_lindex) d.d_lindex = &di;
  if (!d.d_mindex) d.d_mindex = &di;
  return euv_amp_workspace_bytes(&d);
}

int check_run(const euv_plan* P, const uint8_t* d_masks, int n_clips, int n_mask_slices,
              const void* out, const char* who) {
  if (!P || !P->dev) {
    euv_set_error("%s: plan not uploaded (euv_plan_upload)", who);
    return EUV_ERR_BAD_ARG;
  }
  if (!d_masks || !out || n_clips <= 0 || n_clips > P->max_clips ||
      (n_mask_slices != 1 && n_mask_slices != P->cfg.n_slices)) {
    euv_set_error("%s: bad arguments (n_clips %d of at most %d, %d mask slices for %d absorber "
                  "slices)", who, n_clips, P->max_clips, n_mask_slices, P->cfg.n_slices);
    return EUV_ERR_BAD_ARG;
  }
  return EUV_OK;
}

// Spectra of every clip's slices for the order limits lh, mh: d_spec
// [clip][n_slices][(2lh+1)(2mh+1)]; one mask per clip is used for all slices.
struct SpecPlan {
  size_t spec, raw, scratch;  // bytes of each region
};
SpecPlan spec_sizes(const euv_plan* P, int n_masks_total, int n_clips, int n_mask_slices, int lh,
                    int mh) {
  const euv_config& c = P->cfg;
  const size_t S = (size_t)(2 * lh + 1) * (2 * mh + 1);
  SpecPlan s;
  s.spec = (((size_t)n_clips * c.n_slices * S * sizeof(euv_c64)) + 255) & ~(size_t)255;
  s.raw = (n_mask_slices == 1 && c.n_slices > 1)
              ? ((((size_t)n_clips * S * sizeof(euv_c64)) + 255) & ~(size_t)255)
              : 0;
  s.scratch = euv_mask_spectrum_workspace_bytes(n_masks_total, c.ndivx, c.ndivy, P->info.fdivx,
                                                P->info.fdivy, lh, mh);
  return s;
}

int run_spectra(const euv_plan* P, const uint8_t* d_masks, int n_clips, int n_mask_slices, int lh,
                int mh, int select_vacuum, euv_c64* spec, euv_c64* raw, void* scratch,
                size_t scratch_bytes, cudaStream_t stream) {
  const euv_config& c = P->cfg;
  const size_t S = (size_t)(2 * lh + 1) * (2 * mh + 1);
  const bool expand = n_mask_slices == 1 && c.n_slices > 1;
  int rc = euv_mask_spectrum(d_masks, n_clips * n_mask_slices, c.ndivx, c.ndivy, P->info.fdivx,
                             P->info.fdivy, lh, mh, select_vacuum, c.yflip_offset,
                             expand ? raw : spec, scratch, scratch_bytes, stream);
  if (rc) return rc;
  if (expand)
    for (int cl = 0; cl < n_clips; ++cl)
      for (int n = 0; n < c.n_slices; ++n)
        EUV_CUDA_TRY(cudaMemcpyAsync(spec + ((size_t)cl * c.n_slices + n) * S, raw + (size_t)cl * S,
                                     S * sizeof(euv_c64), cudaMemcpyDeviceToDevice, stream));
  return EUV_OK;
}

// ampS of every clip at one incidence for the NA sources, into d_ax
// [clip][nna][N]; the workspace holds the spectra, the unit arrays and the
// ampS scratch.
struct AmpRegions {
  SpecPlan sp;
  size_t units, amp;
  size_t total;
};
AmpRegions amp_regions(const euv_plan* P, int n_clips, int n_mask_slices, euv_amp_desc* dsc) {
  AmpRegions r;
  r.sp = spec_sizes(P, n_clips * n_mask_slices, n_clips, n_mask_slices, 2 * P->info.lmax,
                    2 * P->info.mmax);
  const size_t nna = P->info.n_na_sources;
  Carve cv;
  cv.take<double>(n_clips);
  cv.take<double>(n_clips);
  cv.take<int>(n_clips);
  cv.take<int>(n_clips);
  cv.take<int>((size_t)n_clips * nna);
  cv.take<double>((size_t)n_clips * nna);
  r.units = cv.off;
  euv_amp_desc d = amp_base(P);
  d.n_units = n_clips;
  d.n_src = (int)nna;
  d.k0_max = P->info.k;
  r.amp = euv::amp_bytes(d);
  if (dsc) *dsc = d;
  r.total = r.sp.spec + r.sp.raw + r.units + std::max(r.sp.scratch, r.amp) + 256;
  return r;
}

int run_na_amp(const euv_plan* P, int polar, double kx0, double ky0, const uint8_t* d_masks,
               int n_clips, int n_mask_slices, euv_c64* d_ax, char* w, size_t bytes,
               cudaStream_t stream) {
  euv_amp_desc d;
  AmpRegions r = amp_regions(P, n_clips, n_mask_slices, &d);
  if (bytes < r.total || (reinterpret_cast<uintptr_t>(w) & 255u)) {
    euv_set_error("euv_plan_amp: workspace too small or not 256-byte aligned (%zu < %zu)", bytes,
                  r.total);
    return EUV_ERR_WORKSPACE;
  }
  euv_c64* spec = reinterpret_cast<euv_c64*>(w);
  euv_c64* raw = reinterpret_cast<euv_c64*>(w + r.sp.spec);
  char* u = w + r.sp.spec + r.sp.raw;
  char* scratch = u + r.units;
  const size_t sbytes = bytes - (size_t)(scratch - w);
  const int nna = P->info.n_na_sources;
  Carve cv;
  double* u_kx0 = reinterpret_cast<double*>(u + cv.take<double>(n_clips));
  double* u_ky0 = reinterpret_cast<double*>(u + cv.take<double>(n_clips));
  int* u_pol = reinterpret_cast<int*>(u + cv.take<int>(n_clips));
  int* u_clip = reinterpret_cast<int*>(u + cv.take<int>(n_clips));
  int* u_order = reinterpret_cast<int*>(u + cv.take<int>((size_t)n_clips * nna));
  double* u_kz2 = reinterpret_cast<double*>(u + cv.take<double>((size_t)n_clips * nna));
  int rc = run_spectra(P, d_masks, n_clips, n_mask_slices, 2 * P->info.lmax, 2 * P->info.mmax, 0,
                       spec, raw, scratch, sbytes, stream);
  if (rc) return rc;
  const int tot = n_clips * nna;
  plan_na_units_kernel<<<(tot + 127) / 128, 128, 0, stream>>>(
      n_clips, nna, kx0, ky0, polar, P->info.k, (double)P->cfg.ndivx, (double)P->cfg.ndivy,
      reinterpret_cast<const int*>(P->dev + P->L.na_l),
      reinterpret_cast<const int*>(P->dev + P->L.na_m),
      reinterpret_cast<const int*>(P->dev + P->L.na_order), u_kx0, u_ky0, u_pol, u_clip, u_order,
      u_kz2);
  EUV_LAUNCH_CHECK();
  d.d_kx0 = u_kx0;
  d.d_ky0 = u_ky0;
  d.d_polar = u_pol;
  d.d_spec = u_clip;
  d.d_src_order = u_order;
  d.d_src_2kz = u_kz2;
  d.k0_max = std::max(std::fabs(kx0), std::fabs(ky0));
  return euv_amp(&d, spec, d_ax, scratch, sbytes, stream);
}

}  // namespace
}  // namespace euv

using namespace euv;

extern "C" void euv_config_reference(euv_config* c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  c->ndivx = c->ndivy = 2048;
  c->delta = 1.0;
  c->wavelength = 13.5;
  c->theta0 = -6.0;
  c->azimuth = 0.0;
  c->na = 0.33;
  c->mx = c->my = 4;
  c->illum_type = 1;
  c->sigma1 = 0.9;
  c->sigma2 = 0.55;
  c->openangle = 90.0;
  c->sigmadiv = 0.5;
  c->ndivs = 0;
  c->max_sources = 0;
  c->n_slices = 1;
  // Ta absorber n = 0.9567 + 0.0343i (intensity.cpp:81): eps = n^2
  c->eabs[0] = euv_c64{0.9567 * 0.9567 - 0.0343 * 0.0343, 2.0 * 0.9567 * 0.0343};
  c->dabs[0] = 60.0;
  c->z0_offset = 42.0;
  // multilayer materials and thicknesses (header.h:1217-1230): eps = n^2
  auto sq = [](double re, double im) { return euv_c64{re * re - im * im, 2.0 * re * im}; };
  c->stack.eps_mo = sq(0.9238, 0.006435);
  c->stack.eps_si = sq(0.999, 0.001826);
  c->stack.eps_ru = sq(0.8863, 0.01706);
  c->stack.eps_mosi2 = sq(0.9693, 0.004333);
  c->stack.eps_rusi = sq(0.9099, 0.01547);
  c->stack.eps_sio2 = sq(0.978, 0.01083);
  c->stack.d_mo = 2.052;
  c->stack.d_mosi = 1.661;
  c->stack.d_si = 2.283;
  c->stack.d_simo = 1.045;
  c->stack.d_siru = 0.8;
  c->stack.d_ru = 2.5;
  c->stack.nml = 40;
  c->refresh_sigma = 0;
  c->order_kind = EUV_ORDERS_DIAMOND;
  c->cut = 6.0;
  c->z = 0.0;
  c->yflip_offset = 0;
  c->n_pols = 1;
  c->pols[0] = 0;
  c->pols[1] = 1;
  c->precision = EUV_PREC_FP64;
}

extern "C" int euv_plan_create(const euv_config* cfg, euv_plan** out) {
  if (!cfg || !out) {
    euv_set_error("euv_plan_create: NULL argument");
    return EUV_ERR_BAD_ARG;
  }
  *out = nullptr;
  euv_plan* P = new euv_plan();
  P->cfg = *cfg;
  const int rc = euv::build(P);
  if (rc) {
    delete P;
    return rc;
  }
  *out = P;
  return EUV_OK;
}

extern "C" void euv_plan_destroy(euv_plan* plan) { delete plan; }

extern "C" int euv_plan_get_info(const euv_plan* P, euv_plan_info* info) {
  if (!P || !info) {
    euv_set_error("euv_plan_get_info: NULL argument");
    return EUV_ERR_BAD_ARG;
  }
  *info = P->info;
  return EUV_OK;
}

extern "C" int euv_plan_get_orders(const euv_plan* P, int* h_l, int* h_m) {
  if (!P) return euv::fail("NULL plan");
  if (h_l) std::memcpy(h_l, P->lidx.data(), P->lidx.size() * sizeof(int));
  if (h_m) std::memcpy(h_m, P->midx.data(), P->midx.size() * sizeof(int));
  return EUV_OK;
}

extern "C" int euv_plan_get_pupil(const euv_plan* P, int* h_l, int* h_m, int* h_xinput) {
  if (!P) return euv::fail("NULL plan");
  if (h_l) std::memcpy(h_l, P->lin.data(), P->lin.size() * sizeof(int));
  if (h_m) std::memcpy(h_m, P->min_.data(), P->min_.size() * sizeof(int));
  if (h_xinput) std::memcpy(h_xinput, P->xin.data(), P->xin.size() * sizeof(int));
  return EUV_OK;
}

extern "C" int euv_plan_get_sources(const euv_plan* P, int* h_nsx, int* h_nsy, int* h_count,
                                    int* h_l, int* h_m) {
  if (!P) return euv::fail("NULL plan");
  int o = 0;
  for (size_t f = 0; f < P->fams.size(); ++f) {
    const euv::Fam& F = P->fams[f];
    if (h_nsx) h_nsx[f] = F.nsx;
    if (h_nsy) h_nsy[f] = F.nsy;
    if (h_count) h_count[f] = (int)F.pts.size();
    for (const auto& pt : F.pts) {
      if (h_l) h_l[o] = pt.first;
      if (h_m) h_m[o] = pt.second;
      ++o;
    }
  }
  return EUV_OK;
}

extern "C" int euv_plan_get_na_sources(const euv_plan* P, int* h_l, int* h_m) {
  if (!P) return euv::fail("NULL plan");
  if (h_l) std::memcpy(h_l, P->na_l.data(), P->na_l.size() * sizeof(int));
  if (h_m) std::memcpy(h_m, P->na_m.data(), P->na_m.size() * sizeof(int));
  return EUV_OK;
}

extern "C" int euv_plan_get_abbe_table(const euv_plan* P, int t, euv_c64* h_coef, int* h_nidx) {
  if (!P || t < 0 || t >= P->ntab) return euv::fail("bad plan or table index");
  const size_t per = (size_t)P->n_src * P->info.ncut;
  if (h_coef) std::memcpy(h_coef, P->coef.data() + (size_t)t * per * 3, per * 3 * sizeof(euv_c64));
  if (h_nidx) std::memcpy(h_nidx, P->nidx.data() + (size_t)t * per, per * sizeof(int));
  return EUV_OK;
}

extern "C" size_t euv_plan_device_bytes(const euv_plan* P, int max_clips) {
  if (!P || max_clips <= 0) return 0;
  return euv::layout(P, max_clips).total;
}

extern "C" int euv_plan_upload(euv_plan* P, int max_clips, void* d_tables, size_t bytes,
                               void* stream_) {
  if (!P || max_clips <= 0 || !d_tables || (reinterpret_cast<uintptr_t>(d_tables) & 255u)) {
    euv_set_error("euv_plan_upload: bad arguments (device buffer must be 256-byte aligned)");
    return EUV_ERR_BAD_ARG;
  }
  const euv::DevLayout L = euv::layout(P, max_clips);
  if (bytes < L.total) {
    euv_set_error("euv_plan_upload: buffer too small (%zu < %zu)", bytes, L.total);
    return EUV_ERR_WORKSPACE;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  const euv_plan_info& I = P->info;
  const int ntab = P->ntab, ns = P->n_src, nf = I.n_families;
  std::vector<char>& st = P->staging;
  st.assign(L.total, 0);
  using euv::put;
  put(st, L.lidx, P->lidx.data(), P->lidx.size());
  put(st, L.midx, P->midx.data(), P->midx.size());
  // units u = clip * ntab + t; image of a unit = clip * n_pols + its polarisation
  std::vector<double> kx0, ky0, kz2, invw((size_t)max_clips * I.n_pols, 1.0 / I.sdivsum);
  std::vector<int> pol, clip, order, tab, img, nsrc;
  for (int cl = 0; cl < max_clips; ++cl)
    for (int t = 0; t < ntab; ++t) {
      kx0.push_back(P->tab_kx0[t]);
      ky0.push_back(P->tab_ky0[t]);
      pol.push_back(P->tab_pol[t]);
      clip.push_back(cl);
      for (int s = 0; s < ns; ++s) {
        order.push_back(P->tab_order[(size_t)t * ns + s]);
        kz2.push_back(P->tab_kz2[(size_t)t * ns + s]);
      }
      tab.push_back(t);
      img.push_back(cl * I.n_pols + t / nf);
      nsrc.push_back(P->tab_nsrc[t]);
    }
  put(st, L.u_kx0, kx0.data(), kx0.size());
  put(st, L.u_ky0, ky0.data(), ky0.size());
  put(st, L.u_pol, pol.data(), pol.size());
  put(st, L.u_clip, clip.data(), clip.size());
  put(st, L.u_order, order.data(), order.size());
  put(st, L.u_kz2, kz2.data(), kz2.size());
  put(st, L.u_tab, tab.data(), tab.size());
  put(st, L.u_img, img.data(), img.size());
  put(st, L.u_nsrc, nsrc.data(), nsrc.size());
  put(st, L.inv_w, invw.data(), invw.size());
  put(st, L.coef, P->coef.data(), P->coef.size());
  put(st, L.nidx, P->nidx.data(), P->nidx.size());
  put(st, L.px, P->lin.data(), P->lin.size());
  put(st, L.py, P->min_.data(), P->min_.size());
  put(st, L.row_start, P->row_start.data(), P->row_start.size());
  put(st, L.na_l, P->na_l.data(), P->na_l.size());
  put(st, L.na_m, P->na_m.data(), P->na_m.size());
  put(st, L.na_order, P->na_order.data(), P->na_order.size());
  put(st, L.n_lidx, P->nlidx.data(), P->nlidx.size());
  put(st, L.n_midx, P->nmidx.data(), P->nmidx.size());
  if (P->m3d_error.empty()) {
    // the two narrow solves of m3d.cpp:214-238 (all-vacuum mask = spectrum 0,
    // all-absorber = 1) at the chief-ray incidence, polarisation pols[0]
    const double k = I.k, dx = P->cfg.ndivx, dy = P->cfg.ndivy;
    const double nk[2] = {I.kx0, I.kx0}, nky[2] = {I.ky0, I.ky0};
    const int np_[2] = {P->cfg.pols[0], P->cfg.pols[0]}, nsp[2] = {0, 1};
    const int nna = I.n_na_sources;
    std::vector<int> no(2 * (size_t)nna);
    std::vector<double> nz(2 * (size_t)nna);
    for (int u = 0; u < 2; ++u)
      for (int s = 0; s < nna; ++s) {
        const double kx = I.kx0 + P->na_l[s] * 2.0 * euv::kPi / dx;
        const double ky = I.ky0 + P->na_m[s] * 2.0 * euv::kPi / dy;
        no[(size_t)u * nna + s] = P->src_nn[s];
        nz[(size_t)u * nna + s] = 2.0 * std::sqrt(k * k - kx * kx - ky * ky);
      }
    put(st, L.n_kx0, nk, 2);
    put(st, L.n_ky0, nky, 2);
    put(st, L.n_pol, np_, 2);
    put(st, L.n_spec, nsp, 2);
    put(st, L.n_order, no.data(), no.size());
    put(st, L.n_kz2, nz.data(), nz.size());
    put(st, L.src_nn, P->src_nn.data(), P->src_nn.size());
    put(st, L.pair, P->pair.data(), P->pair.size());
  }
  put(st, L.lin, P->lin.data(), P->lin.size());
  put(st, L.min_, P->min_.data(), P->min_.size());
  put(st, L.xin, P->xin.data(), P->xin.size());
  // the staging copy lives in the plan, so the asynchronous copy may outlast this call
  EUV_CUDA_TRY(cudaMemcpyAsync(d_tables, st.data(), L.total, cudaMemcpyHostToDevice, stream));
  P->dev = reinterpret_cast<char*>(d_tables);
  P->L = L;
  P->max_clips = max_clips;
  P->uniform_done = false;
  return EUV_OK;
}

extern "C" int euv_plan_check(const euv_plan* P, int* bits, void* stream_) {
  if (!P || !P->dev) {
    euv_set_error("euv_plan_check: plan not uploaded");
    return EUV_ERR_BAD_ARG;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  int* d_status = reinterpret_cast<int*>(P->dev + P->L.status);
  int h = 0;
  EUV_CUDA_TRY(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream));
  EUV_CUDA_TRY(cudaStreamSynchronize(stream));
  if (bits) *bits = h;
  if (h) {
    EUV_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int), stream));
    if (h & EUV_STATUS_TIMEOUT) {
      euv_set_error("euv_plan: a bounded device wait gave up (status 0x%x)", h);
      return EUV_ERR_TIMEOUT;
    }
    if (h & EUV_STATUS_SINGULAR) {
      euv_set_error("euv_plan: an LU met a zero pivot (status 0x%x)", h);
      return EUV_ERR_SINGULAR;
    }
    euv_set_error("euv_plan: device status 0x%x", h);
    return EUV_ERR_CUDA;
  }
  return EUV_OK;
}

// ------------------------------------------------------------------ intensity
namespace {
struct IntensityRegions {
  euv::SpecPlan sp;
  size_t ax, amp, total;
};
IntensityRegions intensity_regions(const euv_plan* P, int n_clips, int n_mask_slices,
                                   euv_amp_desc* dsc) {
  IntensityRegions r;
  r.sp = euv::spec_sizes(P, n_clips * n_mask_slices, n_clips, n_mask_slices, 2 * P->info.lmax,
                         2 * P->info.mmax);
  const size_t U = (size_t)n_clips * P->ntab;
  r.ax = ((U * P->n_src * P->info.n_orders * sizeof(euv_c64)) + 255) & ~(size_t)255;
  euv_amp_desc d = euv::amp_base(P);
  d.n_units = (int)U;
  d.n_src = P->n_src;
  d.k0_max = P->info.k;
  r.amp = euv::amp_bytes(d);
  if (dsc) *dsc = d;
  r.total = r.sp.spec + r.sp.raw + r.ax + std::max(r.sp.scratch, r.amp) + 256;
  return r;
}
}  // namespace

extern "C" size_t euv_plan_intensity_workspace_bytes(const euv_plan* P, int n_clips,
                                                     int n_mask_slices) {
  if (!P || n_clips <= 0 || n_mask_slices <= 0) return 0;
  return intensity_regions(P, n_clips, n_mask_slices, nullptr).total;
}

extern "C" int euv_plan_intensity(const euv_plan* P, const uint8_t* d_masks, int n_clips,
                                  int n_mask_slices, double* d_image, void* d_work,
                                  size_t work_bytes, void* stream_) {
  int rc = euv::check_run(P, d_masks, n_clips, n_mask_slices, d_image, "euv_plan_intensity");
  if (rc) return rc;
  cudaStream_t stream = (cudaStream_t)stream_;
  euv_amp_desc d;
  IntensityRegions r = intensity_regions(P, n_clips, n_mask_slices, &d);
  char* w = reinterpret_cast<char*>(d_work);
  if (!w || work_bytes < r.total || (reinterpret_cast<uintptr_t>(w) & 255u)) {
    euv_set_error("euv_plan_intensity: workspace too small or not 256-byte aligned (%zu < %zu)",
                  work_bytes, r.total);
    return EUV_ERR_WORKSPACE;
  }
  euv_c64* spec = reinterpret_cast<euv_c64*>(w);
  euv_c64* raw = reinterpret_cast<euv_c64*>(w + r.sp.spec);
  euv_c64* ax = reinterpret_cast<euv_c64*>(w + r.sp.spec + r.sp.raw);
  char* scratch = w + r.sp.spec + r.sp.raw + r.ax;
  const size_t sbytes = work_bytes - (size_t)(scratch - w);
  if ((rc = euv::run_spectra(P, d_masks, n_clips, n_mask_slices, 2 * P->info.lmax,
                             2 * P->info.mmax, 0, spec, raw, scratch, sbytes, stream)))
    return rc;
  const char* D = P->dev;
  const euv::DevLayout& L = P->L;
  d.d_kx0 = reinterpret_cast<const double*>(D + L.u_kx0);
  d.d_ky0 = reinterpret_cast<const double*>(D + L.u_ky0);
  d.d_polar = reinterpret_cast<const int*>(D + L.u_pol);
  d.d_spec = reinterpret_cast<const int*>(D + L.u_clip);
  d.d_src_order = reinterpret_cast<const int*>(D + L.u_order);
  d.d_src_2kz = reinterpret_cast<const double*>(D + L.u_kz2);
  double k0 = 0.0;
  for (size_t t = 0; t < P->tab_kx0.size(); ++t)
    k0 = std::max(k0, std::max(std::fabs(P->tab_kx0[t]), std::fabs(P->tab_ky0[t])));
  d.k0_max = k0;
  if ((rc = euv_amp(&d, spec, ax, scratch, sbytes, stream))) return rc;
  const euv_plan_info& I = P->info;
  const size_t img = (size_t)n_clips * I.n_pols * I.xdiv * I.ydiv;
  EUV_CUDA_TRY(cudaMemsetAsync(d_image, 0, img * sizeof(double), stream));
  euv_abbe_desc a;
  std::memset(&a, 0, sizeof(a));
  a.xdiv = I.xdiv;
  a.ydiv = I.ydiv;
  a.lpx = I.lpx;
  a.lpy = I.lpy;
  a.ncut = I.ncut;
  a.n_units = n_clips * P->ntab;
  a.n_src = P->n_src;
  a.n_order = I.n_orders;
  a.d_coef = reinterpret_cast<const euv_c64*>(D + L.coef);
  a.d_nidx = reinterpret_cast<const int*>(D + L.nidx);
  a.d_px = reinterpret_cast<const int*>(D + L.px);
  a.d_py = reinterpret_cast<const int*>(D + L.py);
  a.d_row_start = reinterpret_cast<const int*>(D + L.row_start);
  a.d_tab_of_unit = reinterpret_cast<const int*>(D + L.u_tab);
  a.d_img_of_unit = reinterpret_cast<const int*>(D + L.u_img);
  a.d_nsrc_of_unit = reinterpret_cast<const int*>(D + L.u_nsrc);
  a.n_images = n_clips * I.n_pols;
  a.d_inv_weight = reinterpret_cast<const double*>(D + L.inv_w);
  a.precision = P->cfg.precision;
  return euv_abbe(&a, ax, d_image, stream);
}

// ------------------------------------------------------------------ ampS at the NA sources
extern "C" size_t euv_plan_amp_workspace_bytes(const euv_plan* P, int n_clips, int n_mask_slices) {
  if (!P || n_clips <= 0 || n_mask_slices <= 0) return 0;
  return euv::amp_regions(P, n_clips, n_mask_slices, nullptr).total;
}

extern "C" int euv_plan_amp(const euv_plan* P, int polar, double kx0, double ky0,
                            const uint8_t* d_masks, int n_clips, int n_mask_slices, euv_c64* d_ax,
                            void* d_work, size_t work_bytes, void* stream) {
  int rc = euv::check_run(P, d_masks, n_clips, n_mask_slices, d_ax, "euv_plan_amp");
  if (rc) return rc;
  if (polar != 0 && polar != 1) {
    euv_set_error("euv_plan_amp: polar must be 0 (X) or 1 (Y)");
    return EUV_ERR_BAD_ARG;
  }
  for (int s = 0; s < P->info.n_na_sources; ++s)
    if (P->na_order[s] < 0) {
      euv_set_error("euv_plan_amp: the order set misses an NA-circle source order");
      return EUV_ERR_BAD_ARG;
    }
  if (!d_work) {
    euv_set_error("euv_plan_amp: NULL workspace");
    return EUV_ERR_WORKSPACE;
  }
  return euv::run_na_amp(P, polar, kx0, ky0, d_masks, n_clips, n_mask_slices, d_ax,
                         reinterpret_cast<char*>(d_work), work_bytes, (cudaStream_t)stream);
}

// ------------------------------------------------------------------ M3D parameters
namespace {
struct M3dRegions {
  size_t uni_masks, uni_spec, uni_scratch, uni_total;  // narrow solves
  size_t ax_wide, fmask, gather, fspec_scratch, amp_total, total;
};
M3dRegions m3d_regions(const euv_plan* P, int n_clips, int n_mask_slices) {
  const euv_config& c = P->cfg;
  const euv_plan_info& I = P->info;
  M3dRegions r;
  const size_t nb = (size_t)c.ndivx * c.ndivy / 8;
  auto al = [](size_t b) { return (b + 255) & ~(size_t)255; };
  r.uni_masks = al(2 * nb);
  const int lhn = 2 * P->lmax_n, mhn = 2 * P->mmax_n;
  const size_t Sn = (size_t)(2 * lhn + 1) * (2 * mhn + 1);
  r.uni_spec = al(2 * (size_t)c.n_slices * Sn * sizeof(euv_c64)) +
               (c.n_slices > 1 ? al(2 * Sn * sizeof(euv_c64)) : 0);
  euv_amp_desc d = euv::amp_base(P);
  d.n_orders = I.n_orders_narrow;
  d.lmax = P->lmax_n;
  d.mmax = P->mmax_n;
  d.n_units = 2;
  d.n_src = I.n_na_sources;
  d.k0_max = I.k;
  r.uni_scratch = std::max(euv_mask_spectrum_workspace_bytes(2, c.ndivx, c.ndivy, I.fdivx, I.fdivy,
                                                             lhn, mhn),
                           euv::amp_bytes(d));
  r.uni_total = r.uni_masks + r.uni_spec + r.uni_scratch + 256;
  r.ax_wide = al((size_t)n_clips * I.n_na_sources * I.n_orders * sizeof(euv_c64));
  r.fmask = al((size_t)n_clips * (2 * I.lpx + 1) * (2 * I.lpy + 1) * sizeof(euv_c64));
  r.gather = n_mask_slices > 1 ? al((size_t)n_clips * nb) : 0;
  r.fspec_scratch = euv_mask_spectrum_workspace_bytes(n_clips, c.ndivx, c.ndivy, I.fdivx, I.fdivy,
                                                      I.lpx, I.lpy);
  r.amp_total = euv::amp_regions(P, n_clips, n_mask_slices, nullptr).total;
  r.total = std::max(r.uni_total, r.ax_wide + r.fmask + r.gather +
                                       std::max(r.fspec_scratch, r.amp_total) + 256);
  return r;
}
}  // namespace

extern "C" size_t euv_plan_m3d_workspace_bytes(const euv_plan* P, int n_clips, int n_mask_slices) {
  if (!P || n_clips <= 0 || n_mask_slices <= 0) return 0;
  return m3d_regions(P, n_clips, n_mask_slices).total;
}

extern "C" int euv_plan_m3d(euv_plan* P, const uint8_t* d_masks, int n_clips, int n_mask_slices,
                            euv_c64* d_a0, euv_c64* d_ax, euv_c64* d_ay, void* d_work,
                            size_t work_bytes, void* stream_) {
  int rc = euv::check_run(P, d_masks, n_clips, n_mask_slices, d_a0, "euv_plan_m3d");
  if (rc) return rc;
  if (!d_ax || !d_ay) {
    euv_set_error("euv_plan_m3d: NULL output");
    return EUV_ERR_BAD_ARG;
  }
  if (!P->m3d_error.empty()) {
    euv_set_error("euv_plan_m3d: %s", P->m3d_error.c_str());
    return EUV_ERR_BAD_ARG;
  }
  const M3dRegions r = m3d_regions(P, n_clips, n_mask_slices);
  char* w = reinterpret_cast<char*>(d_work);
  if (!w || work_bytes < r.total || (reinterpret_cast<uintptr_t>(w) & 255u)) {
    euv_set_error("euv_plan_m3d: workspace too small or not 256-byte aligned (%zu < %zu)",
                  work_bytes, r.total);
    return EUV_ERR_WORKSPACE;
  }
  cudaStream_t stream = (cudaStream_t)stream_;
  const euv_config& c = P->cfg;
  const euv_plan_info& I = P->info;
  const euv::DevLayout& L = P->L;
  char* D = P->dev;
  const size_t nb = (size_t)c.ndivx * c.ndivy / 8;
  const int nna = I.n_na_sources;
  if (!P->uniform_done) {
    // all-vacuum (bits 1) and all-absorber (bits 0) masks, narrow order set
    uint8_t* um = reinterpret_cast<uint8_t*>(w);
    EUV_CUDA_TRY(cudaMemsetAsync(um, 0xFF, nb, stream));
    EUV_CUDA_TRY(cudaMemsetAsync(um + nb, 0x00, nb, stream));
    const int lhn = 2 * P->lmax_n, mhn = 2 * P->mmax_n;
    const size_t Sn = (size_t)(2 * lhn + 1) * (2 * mhn + 1);
    euv_c64* spec = reinterpret_cast<euv_c64*>(w + r.uni_masks);
    euv_c64* raw = reinterpret_cast<euv_c64*>(
        w + r.uni_masks + (((2 * (size_t)c.n_slices * Sn * sizeof(euv_c64)) + 255) & ~(size_t)255));
    char* scratch = w + r.uni_masks + r.uni_spec;
    const size_t sbytes = work_bytes - (size_t)(scratch - w);
    if ((rc = euv::run_spectra(P, um, 2, 1, lhn, mhn, 0, spec, raw, scratch, sbytes, stream)))
      return rc;
    euv_amp_desc d = euv::amp_base(P);
    d.n_orders = I.n_orders_narrow;
    d.lmax = P->lmax_n;
    d.mmax = P->mmax_n;
    d.d_lindex = reinterpret_cast<const int*>(D + L.n_lidx);
    d.d_mindex = reinterpret_cast<const int*>(D + L.n_midx);
    d.n_units = 2;
    d.d_kx0 = reinterpret_cast<const double*>(D + L.n_kx0);
    d.d_ky0 = reinterpret_cast<const double*>(D + L.n_ky0);
    d.d_polar = reinterpret_cast<const int*>(D + L.n_pol);
    d.d_spec = reinterpret_cast<const int*>(D + L.n_spec);
    d.n_src = nna;
    d.d_src_order = reinterpret_cast<const int*>(D + L.n_order);
    d.d_src_2kz = reinterpret_cast<const double*>(D + L.n_kz2);
    d.k0_max = std::max(std::fabs(I.kx0), std::fabs(I.ky0));
    // ax_vc and ax_ab are the two units of this call, adjacent in the device tables
    if ((rc = euv_amp(&d, spec, reinterpret_cast<euv_c64*>(D + L.ax_vc), scratch, sbytes, stream)))
      return rc;
    P->uniform_done = true;
  }
  // rigorous amplitudes of the clips (wide set, NA sources, chief ray)
  euv_c64* ax_wide = reinterpret_cast<euv_c64*>(w);
  euv_c64* fmask = reinterpret_cast<euv_c64*>(w + r.ax_wide);
  uint8_t* gath = reinterpret_cast<uint8_t*>(w + r.ax_wide + r.fmask);
  char* rest = w + r.ax_wide + r.fmask + r.gather;
  const size_t rbytes = work_bytes - (size_t)(rest - w);
  if ((rc = euv::run_na_amp(P, c.pols[0], I.kx0, I.ky0, d_masks, n_clips, n_mask_slices, ax_wide,
                            rest, rbytes, stream)))
    return rc;
  // thin-mask spectrum of the vacuum indicator of each clip's first slice mask
  const uint8_t* m0 = d_masks;
  if (n_mask_slices > 1) {
    EUV_CUDA_TRY(cudaMemcpy2DAsync(gath, nb, d_masks, nb * n_mask_slices, nb, n_clips,
                                   cudaMemcpyDeviceToDevice, stream));
    m0 = gath;
  }
  if ((rc = euv_mask_spectrum(m0, n_clips, c.ndivx, c.ndivy, I.fdivx, I.fdivy, I.lpx, I.lpy, 1,
                              c.yflip_offset, fmask, rest, rbytes, stream)))
    return rc;
  euv_m3d_desc m;
  std::memset(&m, 0, sizeof(m));
  m.n_clips = n_clips;
  m.n_src = nna;
  m.ninput = I.ncut;
  m.n_order = I.n_orders;
  m.n_order_narrow = I.n_orders_narrow;
  m.lpx = I.lpx;
  m.lpy = I.lpy;
  m.k = I.k;
  m.dx = (double)c.ndivx;
  m.dy = (double)c.ndivy;
  m.z0 = I.z0;
  m.kx0 = I.kx0;
  m.ky0 = I.ky0;
  m.s_center = P->s_center;
  m.d_src_l = reinterpret_cast<const int*>(D + L.na_l);
  m.d_src_m = reinterpret_cast<const int*>(D + L.na_m);
  m.d_src_nidx_narrow = reinterpret_cast<const int*>(D + L.src_nn);
  m.d_ax_vc = reinterpret_cast<const euv_c64*>(D + L.ax_vc);
  m.d_ax_ab = reinterpret_cast<const euv_c64*>(D + L.ax_ab);
  m.d_lin = reinterpret_cast<const int*>(D + L.lin);
  m.d_min = reinterpret_cast<const int*>(D + L.min_);
  m.d_xin = reinterpret_cast<const int*>(D + L.xin);
  m.d_pair_order = reinterpret_cast<const int*>(D + L.pair);
  return euv_m3d_fit(&m, ax_wide, fmask, d_a0, d_ax, d_ay, stream);
}
