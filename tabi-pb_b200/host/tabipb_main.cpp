// tabipb_main.cpp -- host driver mirroring the reference's program TABIPB
// (src/main.f90:11-222) over the C ABI of libtabi_gpu.so.
//
// Run from a directory holding usrdata.in (main.f90:39-50, read positionally
// as "label value" pairs) and test_proteins/<fname>.pqr, exactly like the
// reference's tabipb.exe:
//   readin         readin.f90:2-258   PQR (REAL*4), .xyzr, surface generator
//                                     (tabi_msms with MSMS's flags), .vert/.face,
//                                     surface_area face filter
//   form_matrix    tabi_form_matrix   (main.f90:546-610)
//   treecode_init  tabi_build_tree + the tree-order permutation (main.f90:447-453)
//   DGMRES         tabi_solve         (main.f90:92-139)
//   energy         tabi_energy        (main.f90:144-159)
//   output_potential                  (main.f90:226-326) surface_potential.dat
// Optional trailing usrdata.in lines (ignored by the reference): "tol <v>".
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/tabi_gpu.h"

namespace {

double now() {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void die(const std::string& m) {
  std::fprintf(stderr, "tabipb: %s\n", m.c_str());
  std::exit(1);
}

void check(tabi_h h, int rc, const char* what) {
  if (rc != TABI_OK) die(std::string(what) + " failed: " + tabi_last_error(h));
}

struct UsrData {
  std::string fname, den;
  double eps0 = 1, eps1 = 80, bulk = 0.15, theta = 0.8, tol = 1e-4;
  int order = 3, maxparnode = 500, iprcd = 1, isurf_type = 1;
};

// main.f90:39-50
UsrData read_usrdata(const std::string& path) {
  std::ifstream f(path);
  if (!f) die("cannot open " + path);
  UsrData u;
  std::string label, val;
  std::vector<std::string> vals;
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    if (is >> label >> val) {
      vals.push_back(val);
      if (vals.size() > 10 && label == "tol") u.tol = std::atof(val.c_str());
    }
  }
  if (vals.size() < 10) die("usrdata.in needs 10 label/value lines");
  u.fname = vals[0];
  u.den = vals[1];
  u.eps0 = std::atof(vals[2].c_str());
  u.eps1 = std::atof(vals[3].c_str());
  u.bulk = std::atof(vals[4].c_str());
  u.order = std::atoi(vals[5].c_str());
  u.maxparnode = std::atoi(vals[6].c_str());
  u.theta = std::atof(vals[7].c_str());
  u.iprcd = std::atoi(vals[8].c_str());
  u.isurf_type = std::atoi(vals[9].c_str());
  return u;
}

// readin.f90:29-86: skip REMARK lines; "c1 c2 c3 c4 c5 x y z q r" read as REAL*4
void read_pqr(const std::string& path, std::vector<double>& xyz, std::vector<double>& q,
              std::vector<double>& r) {
  std::ifstream f(path);
  if (!f) die("cannot open " + path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string c[5];
    if (!(is >> c[0])) continue;
    if (c[0].rfind("REMARK", 0) == 0) continue;
    if (c[0].rfind("END", 0) == 0) break;
    if (c[0].rfind("TER", 0) == 0) continue;
    float v[5];
    if (!(is >> c[1] >> c[2] >> c[3] >> c[4] >> v[0] >> v[1] >> v[2] >> v[3] >> v[4])) continue;
    xyz.push_back(v[0]);
    xyz.push_back(v[1]);
    xyz.push_back(v[2]);
    q.push_back(v[3]);
    r.push_back(v[4]);
  }
}

// readin.f90:204-246
void read_msms(const std::string& prefix, std::vector<double>& pos, std::vector<double>& nrm,
               std::vector<int>& face) {
  std::ifstream fv(prefix + ".vert"), ff(prefix + ".face");
  if (!fv || !ff) die("cannot read " + prefix + ".vert/.face");
  std::string line;
  std::getline(fv, line);
  std::getline(fv, line);
  std::getline(fv, line);
  int nspt = std::atoi(line.c_str());
  pos.resize(3 * (size_t)nspt);
  nrm.resize(3 * (size_t)nspt);
  for (int i = 0; i < nspt; ++i) {
    std::getline(fv, line);
    std::istringstream is(line);
    is >> pos[3 * i] >> pos[3 * i + 1] >> pos[3 * i + 2] >> nrm[3 * i] >> nrm[3 * i + 1] >>
        nrm[3 * i + 2];
  }
  std::getline(ff, line);
  std::getline(ff, line);
  std::getline(ff, line);
  int nface = std::atoi(line.c_str());
  face.resize(3 * (size_t)nface);
  for (int i = 0; i < nface; ++i) {
    std::getline(ff, line);
    std::istringstream is(line);
    is >> face[3 * i] >> face[3 * i + 1] >> face[3 * i + 2];
  }
}

double dist3(const double* a, const double* b) {
  double d[3] = {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
  return std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

double heron(double aa, double bb, double cc) {
  double s = 0.5 * (aa + bb + cc);
  return std::sqrt(s * (s - aa) * (s - bb) * (s - cc));
}

// readin.f90:264-333: drop faces with area < 1e-5 or a centroid within squared
// distance 1e-5 of one of the previous 10 faces (of the original list)
double surface_area(const std::vector<double>& pos, std::vector<int>& face) {
  const int nface = (int)face.size() / 3;
  const double third = 1.0 / 3.0;
  std::vector<int> kept;
  double s_area = 0.0;
  std::vector<double> cen(3 * (size_t)nface);
  for (int i = 0; i < nface; ++i) {
    double x[3] = {0, 0, 0};
    for (int j = 0; j < 3; ++j)
      for (int d = 0; d < 3; ++d) x[d] = x[d] + third * pos[3 * (size_t)(face[3 * i + j] - 1) + d];
    for (int d = 0; d < 3; ++d) cen[3 * (size_t)i + d] = x[d];
  }
  for (int i = 0; i < nface; ++i) {
    const double* p0 = &pos[3 * (size_t)(face[3 * i] - 1)];
    const double* p1 = &pos[3 * (size_t)(face[3 * i + 1] - 1)];
    const double* p2 = &pos[3 * (size_t)(face[3 * i + 2] - 1)];
    double a = heron(dist3(p0, p1), dist3(p0, p2), dist3(p1, p2));
    bool alert = false;
    for (int ii = std::max(0, i - 10); ii < i; ++ii) {
      double d[3] = {cen[3 * i] - cen[3 * ii], cen[3 * i + 1] - cen[3 * ii + 1],
                     cen[3 * i + 2] - cen[3 * ii + 2]};
      if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < 1e-5) alert = true;
    }
    if (!(a < 1e-5 || alert))
      for (int j = 0; j < 3; ++j) kept.push_back(face[3 * i + j]);
    s_area += a;
  }
  std::printf(" %d ugly faces are deleted\n", nface - (int)kept.size() / 3);
  face.swap(kept);
  return s_area;
}

}  // namespace

int main(int argc, char** argv) {
  std::string exe_dir = ".";
  {
    std::string a0 = argv[0];
    size_t k = a0.rfind('/');
    if (k != std::string::npos) exe_dir = a0.substr(0, k);
  }
  const std::string msms = argc > 1 ? argv[1] : exe_dir + "/tabi_msms";
  double cpu1 = now();
  UsrData u = read_usrdata("usrdata.in");
  // main.f90:60-65
  const double pi = std::acos(-1.0);
  tabi_params p;
  tabi_default_params(&p);
  p.order = u.order;
  p.maxparnode = u.maxparnode;
  p.theta = u.theta;
  p.kappa = tabi_kappa(u.bulk, u.eps1);
  p.eps0 = u.eps0;
  p.eps1 = u.eps1;
  p.iprcd = u.iprcd;
  p.tol = u.tol;
  const double para = 332.0716;

  // ---- readin
  const std::string base = "test_proteins/" + u.fname;
  std::vector<double> chrpos, atmchr, atmrad;
  read_pqr(base + ".pqr", chrpos, atmchr, atmrad);
  const int nchr = (int)atmchr.size();
  {
    std::ofstream xf(base + ".xyzr");
    char buf[256];
    for (int i = 0; i < nchr; ++i) {
      std::snprintf(buf, sizeof buf, "%.6f %.6f %.6f %.6f\n", chrpos[3 * i], chrpos[3 * i + 1],
                    chrpos[3 * i + 2], atmrad[i]);
      xf << buf;
    }
  }
  if (u.isurf_type != 1)
    std::printf(" isurf_type %d: NanoShaper/ESES are not available; using tabi_msms\n",
                u.isurf_type);
  std::string cmd = msms + " -if " + base + ".xyzr -prob 1.4 -de " + u.den + " -of " + base;
  if (std::system(cmd.c_str()) != 0) die("surface generator failed: " + cmd);
  std::vector<double> sptpos, sptnrm;
  std::vector<int> nvert;
  read_msms(base, sptpos, sptnrm, nvert);
  const int nspt = (int)sptpos.size() / 3;
  std::printf(" # of surfaces= %d  # of surface points= %d\n", (int)nvert.size() / 3, nspt);
  double s_area = surface_area(sptpos, nvert);
  std::printf(" surface area= %g\n", s_area);
  std::remove((base + ".xyzr").c_str());
  std::remove((base + ".vert").c_str());
  std::remove((base + ".face").c_str());
  const int nface = (int)nvert.size() / 3;

  std::printf(" Begin to form linear algebraic matrix...\n");
  double cpu2 = now();
  tabi_h h = nullptr;
  if (tabi_create(&h, &p) != TABI_OK) die(std::string("tabi_create: ") + tabi_last_error(nullptr));
  std::vector<double> tr_xyz(3 * (size_t)nface), tr_q(3 * (size_t)nface), tr_area(nface),
      bvct(2 * (size_t)nface);
  check(h, tabi_form_matrix(h, nspt, sptpos.data(), sptnrm.data(), nface, nvert.data(), nchr,
                            chrpos.data(), atmchr.data(), tr_xyz.data(), tr_q.data(),
                            tr_area.data(), bvct.data()),
        "tabi_form_matrix");
  std::printf(" Begin to initialize treecode...\n");
  std::vector<int> orderarr(nface);
  int nleaf = 0;
  check(h, tabi_build_tree(h, orderarr.data(), &nleaf), "tabi_build_tree");
  std::printf(" number of leaves of the tree: %d\n", nleaf);
  {  // main.f90:443-453
    std::vector<double> tb(bvct), tq(tr_q), ta(tr_area), tx(tr_xyz);
    for (int i = 0; i < nface; ++i) {
      int o = orderarr[i] - 1;
      tr_area[i] = ta[o];
      for (int d = 0; d < 3; ++d) {
        tr_q[3 * i + d] = tq[3 * o + d];
        tr_xyz[3 * i + d] = tx[3 * o + d];
      }
      bvct[i] = tb[o];
      bvct[i + nface] = tb[o + nface];
    }
  }
  double cpu23 = now();
  std::printf(" it takes %g seconds to form the matrix\n", cpu23 - cpu2);
  if (u.iprcd == 1) std::printf(" use block diagonal preconditioning ...\n");
  std::printf(" use msms ...\n Begin to call the solver...\n");

  // ---- DGMRES (main.f90:136-139)
  const int ndim = 2 * nface;
  std::vector<double> xvct(ndim, 0.0), hist((p.nrmax + 1) * p.maxl + 2);
  int iter = 0, ierr = 0, nh = 0;
  double err = 0.0;
  check(h, tabi_solve(h, ndim, bvct.data(), xvct.data(), &iter, &err, &ierr, hist.data(), &nh),
        "tabi_solve");
  for (int k = 0; k < nh; ++k) std::printf(" %10d err= %24.16e\n", k % p.maxl + 1, hist[k]);
  std::printf(" err= %24.16e ierr= %d iter= %d\n", err, ierr, iter);
  double cpu3 = now();

  // ---- energy (main.f90:144-159)
  double soleng = 0.0, couleng = 0.0;
  check(h, tabi_energy(h, nchr, chrpos.data(), atmchr.data(), xvct.data(), &soleng, &couleng),
        "tabi_energy");
  std::printf(" Solvation energy=: %24.16e  kcal/mol\n", soleng);
  std::printf(" -----Free energy=: %24.16e  kcal/mol \n", couleng + soleng);

  // ---- output_potential (main.f90:226-326): on the GPU (tabi_output_potential),
  // the summary prints and the file writer here
  {
    std::vector<double> xo(ndim), vert_ptl(2 * (size_t)nspt);
    check(h, tabi_output_potential(h, nspt, sptpos.data(), nface, nvert.data(), xvct.data(),
                                xo.data(), vert_ptl.data()),
          "tabi_output_potential");
    double emax[4] = {-1e300, -1e300, -1e300, -1e300}, emin[4] = {1e300, 1e300, 1e300, 1e300};
    for (int i = 0; i < nface; ++i) {
      emax[0] = std::max(emax[0], xo[i]);
      emin[0] = std::min(emin[0], xo[i]);
      emax[1] = std::max(emax[1], xo[i + nface]);
      emin[1] = std::min(emin[1], xo[i + nface]);
    }
    for (int i = 0; i < nspt; ++i) {
      emax[2] = std::max(emax[2], vert_ptl[2 * i]);
      emin[2] = std::min(emin[2], vert_ptl[2 * i]);
      emax[3] = std::max(emax[3], vert_ptl[2 * i + 1]);
      emin[3] = std::min(emin[3], vert_ptl[2 * i + 1]);
    }
    std::printf(" The max and min potential and normal derivatives on elements are: \n");
    std::printf(" potential %g %g\n norm derv %g %g\n", emax[0], emin[0], emax[1], emin[1]);
    std::printf(" The max and min potential and normal derivatives on vertices are: \n");
    std::printf(" potential %g %g\n norm derv %g %g\n", emax[2], emin[2], emax[3], emin[3]);
    FILE* fo = std::fopen("surface_potential.dat", "w");
    if (!fo) die("cannot write surface_potential.dat");
    std::fprintf(fo, "%12d%12d\n", nspt, nface);
    for (int i = 0; i < nspt; ++i)
      std::fprintf(fo, "%10d%12.6f%12.6f%12.6f%12.6f%12.6f%12.6f%20.10f%20.10f\n", i + 1,
                   sptpos[3 * i], sptpos[3 * i + 1], sptpos[3 * i + 2], sptnrm[3 * i],
                   sptnrm[3 * i + 1], sptnrm[3 * i + 2], vert_ptl[2 * i], vert_ptl[2 * i + 1]);
    for (int i = 0; i < nface; ++i)
      std::fprintf(fo, "%12d%12d%12d\n", nvert[3 * i], nvert[3 * i + 1], nvert[3 * i + 2]);
    std::fclose(fo);
  }
  double cpu4 = now();
  std::printf(" setup cpu= %g\n solving cpu= %g\n cpu for computing solvation energy= %g\n"
              " Total cpu= %g\n",
              cpu2 - cpu1, cpu3 - cpu2, cpu4 - cpu3, cpu4 - cpu1);
  std::printf(" all done, thank you for using tabipb!\n");
  tabi_destroy(h);
  return ierr == 0 ? 0 : 2;
}
