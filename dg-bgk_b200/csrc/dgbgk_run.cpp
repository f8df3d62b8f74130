// dgbgk_run: the reference's driver on the sm_100a library, one partition.
//
//   dgbgk_run case.con [--precision 64|32] [--device N] [--tol X] [--restart-out] [--parse-only]
//
// Follows src/spectralbgk.f90 (the &Input namelist with its defaults, the
// Lobatto file, the .plt mesh and the FILE.OUT echo), DG_LIN_CONVEC's setup
// (src/dg_lin_convec.f90:70-120: GETSID .. GETNOR, INICON2) and ADVNCE's
// output (src/advnce.f90:103-120, 154-175, 403-435): RESULTS1.RES / RESULTS2.RES
// blocks at step 0, every 1000 steps and after the loop, and one
// RESIDUAL.RES line per step (log of max|DELUN| over the first step's, with
// GETFOR's lift and drag when FORCEOUT != 0, src/getfor.f90).  Files are
// opened by the names the namelist gives, relative to the working directory,
// as the reference does.  RS = 1 starts from RestartInFile in the format
// INICON2 reads (src/inicon2.f90:61-114): a title line, NPOIN and VNPNT,
// then one line per velocity and element (velocity outer) whose first
// three values are DISNF(1:3, IV, IE).
//
// Extensions: --precision 32 stores f in FP32; --tol stops when the L2
// residual falls to tol times the first step's; --restart-out writes the
// final state to RestartOutFile in the format RS = 1 reads (the reference's
// own writer, src/output.f90, is not called by its driver and writes a
// layout its reader does not take); --parse-only prints the parsed inputs as
// JSON and exits (no GPU needed).
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/dgbgk.h"

namespace {

struct Input {
  int TORDER = 20, NTIME = 10000, FORCEOUT = 0, IMMAT = 1, INF = 1, RS = 0, NVSPACEPART = 1;
  double CSAFM = 0.5, rv = 2000, T1 = 293, P1 = 0.1, U0 = 100, V0 = 0, W = 1.0, ALPHA = 0.9, R = 287, d = 250e-12,
         M = 32;
  double CINF[4] = {294, 0.001473, 171.85, 0.0};
  std::string LobattoFile = "Lobatto20.txt", PSpaceFile = "AEROFOIL.RES", OutFile = "FILE.OUT",
              PartitionFile = "METIS3WAYPARTAEROFOIL13.RES", RestartInFile = "RESTART.RES",
              ResidualFile = "RESIDUAL.RES", ResultsFile1 = "RESULTS1.RES", ResultsFile2 = "RESULTS2.RES",
              RestartOutFile = "RESTART.RES", GIDMeshFile = "GIDMESH.RES";
};

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}
std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r\n"), b = s.find_last_not_of(" \t\r\n");
  return a == std::string::npos ? "" : s.substr(a, b - a + 1);
}

// &Input ... / (src/spectralbgk.f90:116-148); gfortran writes strings quoted,
// ifort accepts them bare: both are read.
bool parse_con(const std::string& path, Input& in, std::string& err) {
  std::ifstream fh(path);
  if (!fh) {
    err = "cannot open " + path;
    return false;
  }
  std::string line;
  bool inside = false;
  std::map<std::string, int*> ints = {{"torder", &in.TORDER}, {"ntime", &in.NTIME}, {"forceout", &in.FORCEOUT},
                                      {"immat", &in.IMMAT},   {"inf", &in.INF},     {"rs", &in.RS},
                                      {"nvspacepart", &in.NVSPACEPART}};
  std::map<std::string, double*> reals = {{"csafm", &in.CSAFM}, {"rv", &in.rv}, {"t1", &in.T1}, {"p1", &in.P1},
                                          {"u0", &in.U0},       {"v0", &in.V0}, {"w", &in.W},   {"alpha", &in.ALPHA},
                                          {"r", &in.R},         {"d", &in.d},   {"m", &in.M}};
  std::map<std::string, std::string*> strs = {
      {"lobattofile", &in.LobattoFile},     {"pspacefile", &in.PSpaceFile},       {"outfile", &in.OutFile},
      {"partitionfile", &in.PartitionFile}, {"restartinfile", &in.RestartInFile}, {"residualfile", &in.ResidualFile},
      {"resultsfile1", &in.ResultsFile1},   {"resultsfile2", &in.ResultsFile2},   {"restartoutfile", &in.RestartOutFile},
      {"gidmeshfile", &in.GIDMeshFile}};
  while (std::getline(fh, line)) {
    std::string t = trim(line);
    if (!inside) {
      if (lower(t).rfind("&input", 0) == 0) inside = true;
      continue;
    }
    if (t.rfind("/", 0) == 0) break;
    // the value ends at a '!' comment outside quotes
    std::string body;
    char q = 0;
    for (char c : t) {
      if (q) {
        if (c == q) q = 0;
      } else if (c == '"' || c == '\'') {
        q = c;
      } else if (c == '!') {
        break;
      }
      body += c;
    }
    const size_t eq = body.find('=');
    if (eq == std::string::npos) continue;
    std::string key = lower(trim(body.substr(0, eq))), val = trim(body.substr(eq + 1));
    const size_t pct = key.find('%');
    if (pct != std::string::npos) key = key.substr(pct + 1);
    while (!val.empty() && val.back() == ',') val = trim(val.substr(0, val.size() - 1));
    if (val.size() >= 2 && (val[0] == '"' || val[0] == '\'') && val.back() == val[0]) val = val.substr(1, val.size() - 2);
    int idx = 0;
    const size_t par = key.find('(');
    if (par != std::string::npos) {
      idx = std::atoi(key.c_str() + par + 1);
      key = trim(key.substr(0, par));
    }
    std::string num = val;
    for (auto& c : num)
      if (c == 'd' || c == 'D') c = 'e';
    if (key == "cinf" && idx >= 1 && idx <= 4) {
      in.CINF[idx - 1] = std::strtod(num.c_str(), nullptr);
    } else if (ints.count(key)) {
      *ints[key] = (int)std::lround(std::strtod(num.c_str(), nullptr));
    } else if (reals.count(key)) {
      *reals[key] = std::strtod(num.c_str(), nullptr);
    } else if (strs.count(key)) {
      *strs[key] = val;
    }
  }
  return true;
}

// Fortran 1PE12.5 (a non-finite value is written as gfortran writes it,
// right-aligned NaN / Infinity)
std::string fe12(double x) {
  if (!std::isfinite(x)) {
    std::string r = std::isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity");
    while (r.size() < 12) r = " " + r;
    return r;
  }
  char buf[64];
  std::snprintf(buf, sizeof buf, "%.5E", x);
  std::string s(buf);
  const size_t e = s.find('E');
  const int ex = std::atoi(s.c_str() + e + 1);
  std::string mant = s.substr(0, e);
  char eb[16];
  if (std::abs(ex) < 100)
    std::snprintf(eb, sizeof eb, "E%c%02d", ex < 0 ? '-' : '+', std::abs(ex));
  else
    std::snprintf(eb, sizeof eb, "%c%03d", ex < 0 ? '-' : '+', std::abs(ex));
  std::string r = mant + eb;
  while (r.size() < 12) r = " " + r;
  return r;
}

// the first list-directed token of a line (READ (14,*) TEXT)
std::string first_token(const std::string& line) {
  std::istringstream is(line);
  std::string t;
  is >> t;
  return t;
}
std::string a30(const std::string& s) {
  std::string r = s.substr(0, 30);
  r.resize(30, ' ');
  return r;
}

struct Mesh {
  int nelem = 0, npoin = 0, nboun = 0;
  std::vector<int> intma, bsido;
  std::vector<double> coord;
  std::vector<std::string> echo;  // FILE.OUT lines of the header
};

// The .plt mesh (src/spectralbgk.f90:240-272, src/gtinpt.f90:24-50)
bool read_plt(const std::string& path, Mesh& m, std::string& err) {
  std::ifstream fh(path);
  if (!fh) {
    err = "cannot open the mesh file " + path;
    return false;
  }
  std::string line;
  auto next = [&]() -> bool { return (bool)std::getline(fh, line); };
  if (!next()) return err = "empty mesh file", false;
  const int nlines = std::atoi(first_token(line).c_str());
  for (int i = 0; i < nlines; ++i) {
    if (!next()) return err = "truncated mesh header", false;
    m.echo.push_back(a30(first_token(line)));
  }
  if (!next()) return err = "truncated mesh header", false;
  m.echo.push_back(a30(first_token(line)));
  if (!next()) return err = "truncated mesh header", false;
  const int ndimn = std::atoi(first_token(line).c_str());
  char b6[32];
  std::snprintf(b6, sizeof b6, "%6d", ndimn);
  m.echo.push_back(b6);
  if (ndimn != 2) return err = "only 2-D meshes are supported", false;
  if (!next()) return err = "truncated mesh header", false;
  m.echo.push_back(a30(first_token(line)));
  if (!next()) return err = "truncated mesh header", false;
  {
    std::istringstream is(line);
    is >> m.nelem >> m.npoin >> m.nboun;
  }
  if (m.nelem <= 0 || m.npoin <= 0 || m.nboun < 0) return err = "bad element / point / boundary counts", false;
  char b18[64];
  std::snprintf(b18, sizeof b18, "%6d%6d%6d", m.nelem, m.npoin, m.nboun);
  m.echo.push_back(b18);
  next();  // "connectivities"
  m.intma.resize(3 * (size_t)m.nelem);
  for (int e = 0; e < m.nelem; ++e) {
    if (!next()) return err = "truncated connectivities", false;
    std::istringstream is(line);
    int id;
    is >> id >> m.intma[3 * e] >> m.intma[3 * e + 1] >> m.intma[3 * e + 2];
  }
  next();  // "coordinates"
  m.coord.resize(2 * (size_t)m.npoin);
  for (int p = 0; p < m.npoin; ++p) {
    if (!next()) return err = "truncated coordinates", false;
    for (auto& c : line)
      if (c == 'd' || c == 'D') c = 'e';
    std::istringstream is(line);
    int id;
    is >> id >> m.coord[2 * p] >> m.coord[2 * p + 1];
  }
  next();  // "boundary sides"
  m.bsido.resize(6 * (size_t)m.nboun);
  for (int b = 0; b < m.nboun; ++b) {
    if (!next()) return err = "truncated boundary sides", false;
    std::istringstream is(line);
    for (int k = 0; k < 6; ++k) is >> m.bsido[6 * b + k];
  }
  return true;
}

bool read_lobatto(const std::string& path, std::vector<double>& eta, std::vector<double>& w, std::string& err) {
  std::ifstream fh(path);
  if (!fh) return err = "cannot open the Lobatto file " + path, false;
  std::string tok;
  fh >> tok;
  const double nd = std::strtod(tok.c_str(), nullptr);
  if (!(nd >= 1.0 && nd <= 1.0e6)) return err = "bad point count in the Lobatto file " + path, false;
  const int n = (int)std::lround(nd);
  eta.resize(n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    std::string a, b;
    if (!(fh >> a >> b)) return err = "truncated Lobatto file", false;
    for (auto* s : {&a, &b})
      for (auto& c : *s)
        if (c == 'd' || c == 'D') c = 'e';
    eta[i] = std::strtod(a.c_str(), nullptr);
    w[i] = std::strtod(b.c_str(), nullptr);
  }
  return true;
}

int die(const std::string& msg) {
  std::fprintf(stderr, "dgbgk_run: %s\n", msg.c_str());
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  std::string con;
  int precision = 64, device = 0;
  double tol = 0.0;
  bool parse_only = false, restart_out = false;
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    if (a == "--precision" && i + 1 < argc)
      precision = std::atoi(argv[++i]);
    else if (a == "--device" && i + 1 < argc)
      device = std::atoi(argv[++i]);
    else if (a == "--tol" && i + 1 < argc)
      tol = std::atof(argv[++i]);
    else if (a == "--parse-only")
      parse_only = true;
    else if (a == "--restart-out")
      restart_out = true;
    else if (con.empty())
      con = a;
    else
      return die("unexpected argument " + a);
  }
  if (con.empty())
    return die("usage: dgbgk_run case.con [--precision 64|32] [--device N] [--tol X] [--restart-out] [--parse-only]");
  Input in;
  std::string err;
  if (!parse_con(con, in, err)) return die(err);
  if (parse_only) {
    std::printf("{\"TORDER\": %d, \"NTIME\": %d, \"FORCEOUT\": %d, \"IMMAT\": %d, \"INF\": %d, \"RS\": %d, "
                "\"NVSPACEPART\": %d, \"CSAFM\": %.17g, \"rv\": %.17g, \"T1\": %.17g, \"P1\": %.17g, \"U0\": %.17g, "
                "\"V0\": %.17g, \"W\": %.17g, \"ALPHA\": %.17g, \"R\": %.17g, \"d\": %.17g, \"M\": %.17g, "
                "\"CINF\": [%.17g, %.17g, %.17g, %.17g], \"LobattoFile\": \"%s\", \"PSpaceFile\": \"%s\", "
                "\"OutFile\": \"%s\", \"ResidualFile\": \"%s\", \"ResultsFile1\": \"%s\", \"ResultsFile2\": \"%s\"}\n",
                in.TORDER, in.NTIME, in.FORCEOUT, in.IMMAT, in.INF, in.RS, in.NVSPACEPART, in.CSAFM, in.rv, in.T1,
                in.P1, in.U0, in.V0, in.W, in.ALPHA, in.R, in.d, in.M, in.CINF[0], in.CINF[1], in.CINF[2], in.CINF[3],
                in.LobattoFile.c_str(), in.PSpaceFile.c_str(), in.OutFile.c_str(), in.ResidualFile.c_str(),
                in.ResultsFile1.c_str(), in.ResultsFile2.c_str());
    return 0;
  }

  // velocity space (src/spectralbgk.f90:156-161, src/vspace.f90)
  std::vector<double> eta, wl;
  if (!read_lobatto(in.LobattoFile, eta, wl, err)) return die(err);
  const int RORDER = (int)eta.size(), TORDER = in.TORDER, V = RORDER * TORDER;
  std::vector<double> vcord(3 * (size_t)V);
  double sumweight = 0;
  if (dgbgk_vspace_build(RORDER, TORDER, eta.data(), wl.data(), vcord.data(), &sumweight) != 0)
    return die(dgbgk_last_error());

  // mesh and FILE.OUT (src/spectralbgk.f90:212-272)
  Mesh m;
  if (!read_plt(in.PSpaceFile, m, err)) return die(err);
  {
    FILE* fo = std::fopen(in.OutFile.c_str(), "w");
    if (!fo) return die("cannot write " + in.OutFile);
    for (const auto& l : m.echo) std::fprintf(fo, "%s\n", l.c_str());
    std::fprintf(fo, "V-SPACE STATS:\n");
    std::fprintf(fo, "LOBATTO ORDER      TOTAL NUMBER OF NODES\n");
    std::fprintf(fo, "%6d%6d%6d\n", RORDER, TORDER, V);
    std::fclose(fo);
  }

  // INICON2's restart input, read (and checked) before any device work
  std::vector<double> disnf0;
  if (in.RS == 1) {
    disnf0.assign(3 * (size_t)V * m.nelem, 0.0);
    // INICON2's restart branch (src/inicon2.f90:61-114)
    std::ifstream rf(in.RestartInFile);
    if (!rf) return die("cannot open the restart file " + in.RestartInFile);
    std::string l1, l2;
    std::getline(rf, l1);
    std::getline(rf, l2);
    long long t1 = -1, t2 = -1;
    {
      std::istringstream is(l2);
      is >> t1 >> t2;
    }
    if (t1 != m.npoin || t2 != V) return die("THIS RESTART FILE IS NOT COMPATIBLE WITH YOUR MESHES!");
    std::string line;
    for (int iv = 0; iv < V; ++iv)
      for (int ie = 0; ie < m.nelem; ++ie) {
        // list-directed READ of three values: the first three of the record
        int got = 0;
        double vals[3];
        while (got < 3 && std::getline(rf, line)) {
          for (auto& c : line)
            if (c == 'd' || c == 'D') c = 'e';
          std::istringstream is(line);
          double x;
          while (got < 3 && (is >> x)) vals[got++] = x;
        }
        if (got < 3) return die("truncated restart file " + in.RestartInFile);
        for (int k = 0; k < 3; ++k) disnf0[(size_t)k + 3 * ((size_t)iv + (size_t)V * ie)] = vals[k];
      }
  }

  // setup (src/dg_lin_convec.f90:70-89)
  const int mxsid = 2 * (m.nelem + m.nboun);
  std::vector<int> iside(8 * (size_t)mxsid);
  std::vector<double> nx(mxsid), ny(mxsid), el(mxsid), geome(7 * (size_t)m.nelem), relen(m.nelem),
      mmat(3 * (size_t)m.nelem), cmmat(9 * (size_t)m.nelem), rsido(3 * (size_t)std::max(m.nboun, 1));
  int nside = 0;
  if (dgbgk_setup_mesh(m.nelem, m.npoin, m.nboun, m.intma.data(), m.coord.data(), m.bsido.data(), &nside,
                       iside.data(), nx.data(), ny.data(), el.data(), geome.data(), relen.data(), mmat.data(),
                       cmmat.data(), rsido.data()) != 0)
    return die(dgbgk_last_error());
  dgbgk_mesh dm{m.nelem,        m.npoin,      m.nboun,   nside,     m.intma.data(), m.coord.data(),
                m.bsido.data(), iside.data(), nx.data(), ny.data(), el.data(),      geome.data(),
                relen.data(),   mmat.data(),  cmmat.data(), rsido.data()};
  dgbgk_vspace vs{RORDER, TORDER, vcord.data(), sumweight, in.rv};
  dgbgk_params p;
  dgbgk_default_params(&p);
  p.immat = in.IMMAT;
  p.csafm = in.CSAFM;
  p.alpha = in.ALPHA;
  p.rgas = in.R;
  p.molar_mass = in.M;
  p.diameter = in.d;
  for (int k = 0; k < 4; ++k) p.cinf[k] = in.INF == 1 ? in.CINF[k] : 0.0;  // src/inicon2.f90:185-193
  p.precision = precision;
  p.device = device;
  dgbgk_handle* h = nullptr;
  if (dgbgk_create(&dm, &vs, &p, &h) != 0) return die(dgbgk_last_error());
  if (in.RS == 1) {
    if (dgbgk_set_state(h, disnf0.data()) != 0) return die(dgbgk_last_error());
  } else {
    // INICON2 (src/inicon2.f90:120-182)
    if (dgbgk_init_uniform(h, in.T1, in.P1, in.U0, in.V0, nullptr) != 0) return die(dgbgk_last_error());
  }

  FILE* f16 = std::fopen(in.ResidualFile.c_str(), "w");
  FILE* f17 = std::fopen(in.ResultsFile1.c_str(), "w");
  FILE* f18 = std::fopen(in.ResultsFile2.c_str(), "w");
  if (!f16 || !f17 || !f18) return die("cannot open the output files");
  const int NP = m.npoin;
  std::vector<double> nd(NP), rho(NP), u(NP), v(NP), ps(NP), temp(NP);
  auto gather = [&]() { return dgbgk_get_macros(h, nd.data(), rho.data(), u.data(), v.data(), ps.data(), temp.data()); };
  auto results = [&](int itime) {
    std::fprintf(f17, "RESULTS        1   %5d    2      1      0\n", itime);
    std::fprintf(f18, "RESULTS        1   %5d    2      1      0\n", itime);
    for (int i = 0; i < NP; ++i) {
      std::fprintf(f17, "%5d    %s %s %s \n", i + 1, fe12(nd[i]).c_str(), fe12(u[i]).c_str(), fe12(v[i]).c_str());
      std::fprintf(f18, "%5d    %s %s %s \n", i + 1, fe12(rho[i]).c_str(), fe12(ps[i]).c_str(), fe12(temp[i]).c_str());
    }
  };
  if (gather() != 0) return die(dgbgk_last_error());
  results(0);
  // GETFOR (src/getfor.f90:29-49) on the device
  double lift = 0, drag = 0;
  if (in.FORCEOUT != 0 && dgbgk_get_forces(h, &lift, &drag) != 0) return die(dgbgk_last_error());

  // The time loop.  ADVNCE gathers GETMAC's fields (and GETFOR reads their
  // PS) at MOD(ITIME,1000) = 0 (src/advnce.f90:403-435): the library records
  // them on the device at those steps, and the driver writes them after each
  // advance call of up to kCap such records.
  constexpr int kEvery = 1000, kCap = 8;
  if (dgbgk_set_output(h, kEvery, kCap) != 0) return die(dgbgk_last_error());
  struct Rec {
    int itime = -1;
    double lift = 0, drag = 0;
    std::vector<double> f[6];
  };
  std::vector<Rec> recs(kCap);
  for (auto& r : recs)
    for (auto& x : r.f) x.resize(NP);
  double sritm1 = 0;
  int itime = 0, taken = 0;
  bool stopped = false;
  std::vector<double> linf, l2, dte;
  while (itime < in.NTIME && !stopped) {
    const int n = std::min(in.NTIME - itime, kEvery * kCap);
    linf.resize(n);
    l2.resize(n);
    dte.resize(n);
    int done = 0;
    const int rc = dgbgk_advance(h, n, tol, &done, linf.data(), l2.data(), dte.data());
    if (rc != 0) {
      std::fclose(f16);
      std::fclose(f17);
      std::fclose(f18);
      return die(dgbgk_last_error());
    }
    // this call's records (at most kCap: n <= kEvery * kCap), oldest first
    int count = 0;
    if (dgbgk_output_count(h, &count) != 0) return die(dgbgk_last_error());
    const int fresh = count - taken, held = std::min(count, kCap);
    taken = count;
    for (int r = 0; r < fresh; ++r) {
      Rec& x = recs[r];
      if (dgbgk_get_output(h, held - fresh + r, &x.itime, x.f[0].data(), x.f[1].data(), x.f[2].data(),
                           x.f[3].data(), x.f[4].data(), x.f[5].data(), &x.lift, &x.drag) != 0)
        return die(dgbgk_last_error());
    }
    int next = 0;
    for (int k = 0; k < done; ++k) {
      const int it = itime + k + 1;
      if (next < fresh && it == recs[next].itime) {  // GETMAC before the residual line of the same step
        const Rec& x = recs[next++];
        nd = x.f[0];
        rho = x.f[1];
        u = x.f[2];
        v = x.f[3];
        ps = x.f[4];
        temp = x.f[5];
        results(it);
        lift = x.lift;
        drag = x.drag;
      }
      const double sumres = linf[k];
      if (it == 1) sritm1 = sumres;
      const double lr = std::log(sumres / sritm1);
      if (in.FORCEOUT == 0)
        std::fprintf(f16, "%12d %16.8E\n", it, lr);
      else
        std::fprintf(f16, "%12d %16.8E %16.8E %16.8E\n", it, lr, lift, drag);
    }
    itime += done;
    if (done < n) stopped = true;  // the L2 tolerance was reached
  }
  // after the loop: the last gathered fields under ITIME = NTIME + 1 (the DO
  // variable's value after the loop, src/advnce.f90:482-489)
  results(stopped ? itime + 1 : in.NTIME + 1);
  std::fclose(f16);
  std::fclose(f17);
  std::fclose(f18);
  if (restart_out) {
    std::vector<double> disnf(3 * (size_t)V * m.nelem);
    if (dgbgk_get_state(h, disnf.data()) != 0) return die(dgbgk_last_error());
    FILE* fr = std::fopen(in.RestartOutFile.c_str(), "w");
    if (!fr) return die("cannot write " + in.RestartOutFile);
    std::fprintf(fr, "NPOIN     VNPNT\n%12d    %12d\n", m.npoin, V);
    for (int iv = 0; iv < V; ++iv)
      for (int ie = 0; ie < m.nelem; ++ie) {
        const double* q = &disnf[3 * ((size_t)iv + (size_t)V * ie)];
        std::fprintf(fr, "%.17E %.17E %.17E\n", q[0], q[1], q[2]);
      }
    std::fclose(fr);
  }
  std::printf("dgbgk_run: %d steps of %d elements x %d velocities (FP%d)%s\n", itime, m.nelem, V, precision,
              stopped ? ", stopped at the L2 tolerance" : "");
  dgbgk_destroy(h);
  return 0;
}
