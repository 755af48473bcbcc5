// ecogen-b200: command-line driver with ECOGEN's interface, built on the C ABI.
//
//   ecogen-b200 <work folder>
//
// Like the reference's main (src/main.cpp:44-133) it reads <work>/ECOGEN.xml, runs each <testCase>
// folder in turn with the EOS files of <work>/libEOS, and writes results to
// <work>/results/<run>/: infoCalcul.out (CPU count, then file number, iteration, time, next dt and
// computation seconds per print, src/InputOutput/Output.cpp:491) and, at every print time,
// datasets/result[B64]_CPU0_TIME<k>.vtr — a VTK rectilinear grid with Float64 cell arrays named and
// ordered like the reference's writer (src/InputOutput/OutputXML.cpp:320-470), base64 or ASCII with
// the outputMode precision.  Print control follows Run::solver (src/Run.cpp:417-428): every iterFreq
// iterations, or every timeFreq of physical time and at the end.  <restartSimulation
// restartFileNumber="N"> restarts from result file N and its infoCalcul.out line (Run::restartSimulation
// src/Run.cpp:345, Output::readInfos src/InputOutput/Output.cpp:524): ASCII files as the reference
// reads them, and base64 files too.  A case the library does not run is reported and skipped; the
// exit code is the number of failed cases.
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

extern "C" {
#include "../../include/ecogen_b200.h"
}
#include "ecg_internal.h"  // axis_cells: the mesh's cell sizes and centres

namespace {

std::string b64(const unsigned char* d, size_t n) {
  static const char* tbl = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
  std::string out;
  out.reserve((n + 2) / 3 * 4);
  size_t i = 0;
  for (; i + 2 < n; i += 3) {
    unsigned v = (d[i] << 16) | (d[i + 1] << 8) | d[i + 2];
    out += tbl[(v >> 18) & 63];
    out += tbl[(v >> 12) & 63];
    out += tbl[(v >> 6) & 63];
    out += tbl[v & 63];
  }
  if (i < n) {
    unsigned v = d[i] << 16;
    if (i + 1 < n) v |= d[i + 1] << 8;
    out += tbl[(v >> 18) & 63];
    out += tbl[(v >> 12) & 63];
    out += (i + 1 < n) ? tbl[(v >> 6) & 63] : '=';
    out += '=';
  }
  return out;
}

// VTK inline array.  "binary": base64 of a 4-byte length header, then base64 of the data
// (IO::writeb64Chaine src/InputOutput/IO.cpp:40); "ascii": every value streamed with the stream's
// precision and a space (Output::writeDataset src/InputOutput/Output.cpp:372).
void write_array(std::ostream& f, const std::string& name, const std::vector<double>& v, int ncomp, bool binary) {
  f << "        <DataArray type=\"Float64\"";
  if (!name.empty()) f << " Name=\"" << name << "\"";
  if (ncomp > 1) f << " NumberOfComponents=\"" << ncomp << "\"";
  f << " format=\"" << (binary ? "binary" : "ascii") << "\">\n";
  if (binary) {
    int32_t nb = (int32_t)(v.size() * sizeof(double));
    f << b64(reinterpret_cast<const unsigned char*>(&nb), 4)
      << b64(reinterpret_cast<const unsigned char*>(v.data()), v.size() * sizeof(double)) << "\n";
  } else {
    for (double x : v) f << x << " ";
    f << "\n";
  }
  f << "        </DataArray>\n";
}

int b64val(char ch) {
  if (ch >= 'A' && ch <= 'Z') return ch - 'A';
  if (ch >= 'a' && ch <= 'z') return ch - 'a' + 26;
  if (ch >= '0' && ch <= '9') return ch - '0' + 52;
  if (ch == '+') return 62;
  if (ch == '/') return 63;
  return -1;
}

// Decodes one base64 group sequence (stops at padding); returns false on a bad character.
bool unb64(const std::string& s, size_t pos, size_t len, std::vector<unsigned char>& out) {
  unsigned acc = 0;
  int bits = 0;
  for (size_t i = pos; i < pos + len && i < s.size(); i++) {
    char ch = s[i];
    if (ch == '=') break;
    int v = b64val(ch);
    if (v < 0) return false;
    acc = (acc << 6) | (unsigned)v;
    bits += 6;
    if (bits >= 8) {
      bits -= 8;
      out.push_back((unsigned char)((acc >> bits) & 0xFF));
    }
  }
  return true;
}

// The Float64 cell arrays of a result file, in document order (OutputXML::ReadPhysicalDataXML
// src/InputOutput/OutputXML.cpp:194 reads them by position, not by name).
bool read_cell_arrays(const std::string& path, std::vector<std::vector<double>>& arrays, std::string* err) {
  std::ifstream f(path);
  if (!f) {
    *err = "cannot open " + path;
    return false;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string txt = ss.str();
  size_t pos = txt.find("<CellData>");
  if (pos == std::string::npos) {
    *err = path + ": <CellData> missing";
    return false;
  }
  const size_t end = txt.find("</CellData>", pos);
  while (true) {
    size_t a = txt.find("<DataArray", pos);
    if (a == std::string::npos || (end != std::string::npos && a > end)) break;
    size_t gt = txt.find('>', a);
    size_t close = txt.find("</DataArray>", gt);
    if (gt == std::string::npos || close == std::string::npos) {
      *err = path + ": unterminated DataArray";
      return false;
    }
    const std::string head = txt.substr(a, gt - a);
    std::vector<double> v;
    if (head.find("format=\"binary\"") != std::string::npos) {
      size_t p0 = txt.find_first_not_of(" \t\r\n", gt + 1);
      std::vector<unsigned char> h;
      if (p0 == std::string::npos || !unb64(txt, p0, 8, h) || h.size() < 4) {
        *err = path + ": bad base64 header";
        return false;
      }
      int32_t nb;
      std::memcpy(&nb, h.data(), 4);
      std::vector<unsigned char> d;
      size_t p1 = p0 + 8, p2 = txt.find_last_not_of(" \t\r\n", close - 1);
      if (!unb64(txt, p1, p2 + 1 - p1, d) || nb < 0 || d.size() < (size_t)nb) {
        *err = path + ": bad base64 data";
        return false;
      }
      v.resize((size_t)nb / sizeof(double));
      std::memcpy(v.data(), d.data(), v.size() * sizeof(double));
    } else {
      const char* q = txt.c_str() + gt + 1;
      const char* qe = txt.c_str() + close;
      while (q < qe) {
        char* nx = nullptr;
        double x = std::strtod(q, &nx);
        if (nx == q) break;
        v.push_back(x);
        q = nx;
      }
    }
    arrays.push_back(std::move(v));
    pos = close + 12;
  }
  return true;
}

bool mkdirs(const std::string& p) {
  std::string cur;
  std::stringstream ss(p);
  std::string part;
  if (!p.empty() && p[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part + "/";
    if (mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return false;
  }
  return true;
}

std::string strip_xml(const std::string& s) {  // "SG_water.xml" -> "SG_water" (OutputXML.cpp:430)
  return s.size() > 4 ? s.substr(0, s.size() - 4) : s;
}

std::string result_name(bool binary, int file) {  // OutputXML::createFilenameXML :271
  return std::string("result") + (binary ? "B64" : "") + "_CPU0_TIME" + std::to_string(file) + ".vtr";
}

// |grad rho| of the mixture density by GradientFiniteDifference::computeGradients
// (src/Gradients/GradientFiniteDifference.cpp:46-130, the default gradient method) as
// Cell::getDensityGradient (src/Order1/Cell.cpp:627) evaluates it for the output: each internal face
// of a cell adds n * (rho_R - rho_L) / |x_R - x_L| * |component distance| in the cell's face order
// (x faces, y faces, z faces; minus side first), boundary faces only add twice their centre-to-face
// distance to the normalising sums.
std::vector<double> grad_rho(const ecg_case& c, const std::vector<double>& rho) {
  const int nx = c.ncells[0], ny = c.ncells[1], nz = c.ncells[2];
  const int64_t n = (int64_t)nx * ny * nz;
  const int nn[3] = {nx, ny, nz};
  double bm[3], bp[3];
  std::vector<double> sz[3], ctr[3];  // cell sizes and centres per axis (stretched or uniform)
  for (int a = 0; a < 3; a++) {
    ecg::axis_cells(c, a, sz[a], ctr[a]);
    const double p0 = ctr[a][0], pl = ctr[a][nn[a] - 1];
    bm[a] = std::fabs(p0 - 0.) * 2.;                         // Xm face at 0
    bp[a] = std::fabs(pl - (pl + 0.5 * sz[a][nn[a] - 1])) * 2.;  // Xp face at the last centre + its half size
  }
  std::vector<double> g((size_t)n);
  const int64_t stride[3] = {1, nx, (int64_t)nx * ny};
  for (int64_t i = 0; i < n; i++) {
    const int ijk[3] = {(int)(i % nx), (int)((i / nx) % ny), (int)(i / ((int64_t)nx * ny))};
    double gr[3] = {0., 0., 0.}, sum[3] = {0., 0., 0.};
    for (int a = 0; a < 3; a++) {
      if (nn[a] == 1) continue;
      for (int side = 0; side < 2; side++) {  // face with the previous cell, then with the next one
        const int o = side ? ijk[a] + 1 : ijk[a] - 1;
        if (o < 0 || o >= nn[a]) continue;
        const int64_t L = side ? i : i - stride[a], R = side ? i + stride[a] : i;
        const int iL = side ? ijk[a] : o, iR = side ? o : ijk[a];
        const double xL = ctr[a][iL], xR = ctr[a][iR];
        const double dist_a = std::fabs(xL - xR);
        const double dist = std::sqrt((xL - xR) * (xL - xR) + 0. * 0. + 0. * 0.);
        sum[a] += dist_a;
        const double gf = (rho[R] - rho[L]) / dist;
        for (int b = 0; b < 3; b++) gr[b] = gr[b] + (b == a ? 1. : 0.) * gf * (b == a ? dist_a : 0.);
      }
    }
    for (int a = 0; a < 3; a++) {  // boundary faces: Xm, Xp, Ym, Yp, Zm, Zp
      if (nn[a] == 1) continue;
      if (ijk[a] == 0) sum[a] += bm[a];
      if (ijk[a] == nn[a] - 1) sum[a] += bp[a];
    }
    for (int a = 0; a < 3; a++)
      if (sum[a] <= 1.e-12) sum[a] = 1.;
    const double x = gr[0] / sum[0], y = gr[1] / sum[1], z = gr[2] / sum[2];
    g[i] = std::sqrt(x * x + y * y + z * z);
  }
  return g;
}

// Number of field pointers of the ABI layout (include/ecogen_b200.h).
int abi_fields(const ecg_case& c) {
  if (c.model == ECG_MODEL_EULER) return 6 + c.ntransports;
  if (c.model == ECG_MODEL_PTUEQ) return 2 * c.nphases + 6 + c.ntransports;
  return 2 * c.nphases + 5 + c.ntransports;
}

struct Output {
  std::string dir;
  const ecg_input* in;
  ecg_case c;
  int64_t n;
  int file = 0;
  bool binary = true;
  int precision = 0;

  // Passive transports T1, T2, ..., values below 1e-20 written as 0 (MeshCartesian::getData
  // src/Meshes/MeshCartesian.cpp:1832-1836).
  void write_transports(std::ostream& o, const std::vector<std::vector<double>>& f, int first) {
    for (int j = 0; j < c.ntransports; j++) {
      std::vector<double> v = f[first + j];
      for (double& x : v)
        if (x < 1.e-20) x = 0.;
      write_array(o, "T" + std::to_string(j + 1), v, 1, binary);
    }
  }

  bool write(ecg_ctx* ctx) {
    const int np = c.nphases;
    const bool euler = c.model == ECG_MODEL_EULER;
    const int nf = abi_fields(c);
    std::vector<std::vector<double>> f(nf, std::vector<double>((size_t)n));
    std::vector<double*> ptr;
    for (auto& v : f) ptr.push_back(v.data());
    if (ecg_download_prim(ctx, ptr.data(), n) != ECG_OK) return false;
    std::vector<double> T((size_t)np * n), Y((size_t)np * n);
    if (ecg_download_derived(ctx, T.data(), Y.data(), n) != ECG_OK) return false;
    std::ofstream o(dir + "datasets/" + result_name(binary, file++), std::ios::trunc);
    if (!o) return false;
    if (precision != 0) o.precision(precision);
    int nx = c.ncells[0], ny = c.ncells[1], nz = c.ncells[2];
    o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"RectilinearGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    o << "  <RectilinearGrid WholeExtent=\"0 " << nx << " 0 " << ny << " 0 " << nz << "\">\n";
    o << "    <Piece Extent=\"0 " << nx << " 0 " << ny << " 0 " << nz << "\">\n      <Coordinates>\n";
    for (int a = 0; a < 3; a++) {  // MeshCartesian::getCoord src/Meshes/MeshCartesian.cpp:1791-1815
      std::vector<double> sz, ctr, x;
      ecg::axis_cells(c, a, sz, ctr);
      for (int i = 0; i < c.ncells[a]; i++) x.push_back(ctr[i] - 0.5 * sz[i]);
      x.push_back(ctr[c.ncells[a] - 1] + 0.5 * sz[c.ncells[a] - 1]);
      write_array(o, "", x, 1, binary);
    }
    o << "      </Coordinates>\n      <CellData>\n";
    auto slice = [&](const std::vector<double>& v, int k) {
      return std::vector<double>(v.begin() + (size_t)k * n, v.begin() + (size_t)(k + 1) * n);
    };
    if (euler) {
      std::string e = strip_xml(ecg_input_eos_name(in, 0));
      write_array(o, "F0_Density_" + e, f[0], 1, binary);
      write_array(o, "F0_Pressure_" + e, f[1], 1, binary);
      write_array(o, "F0_Temperature_" + e, slice(T, 0), 1, binary);
      std::vector<double> u((size_t)3 * n);
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) u[3 * i + d] = f[2 + d][i];
      write_array(o, "F0_Velocity_" + e, u, 3, binary);
      write_transports(o, f, 6);
      write_array(o, "gradRho", grad_rho(c, f[0]), 1, binary);
    } else if (c.model == ECG_MODEL_PTUEQ) {
      // PhasePTUEq scalars Alpha, Density (src/Models/PTUEq/PhasePTUEq.cpp:118-150, no display clamp) and
      // MixPTUEq scalars Density, Pressure, Temperature and vector Velocity (MixPTUEq.cpp:236-270)
      for (int k = 0; k < np; k++) {
        std::string e = strip_xml(ecg_input_eos_name(in, k));
        write_array(o, "F" + std::to_string(k) + "_Alpha_" + e, f[k], 1, binary);
        write_array(o, "F" + std::to_string(k) + "_Density_" + e, f[np + k], 1, binary);
      }
      std::vector<double> rho((size_t)n, 0.);
      for (int k = 0; k < np; k++)
        for (int64_t i = 0; i < n; i++) rho[i] += f[k][i] * f[np + k][i];
      write_array(o, "Density_Mixture", rho, 1, binary);
      write_array(o, "Pressure_Mixture", f[2 * np], 1, binary);
      write_array(o, "Temperature_Mixture", f[2 * np + 5], 1, binary);
      std::vector<double> u((size_t)3 * n);
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) u[3 * i + d] = f[2 * np + 1 + d][i];
      write_array(o, "Velocity_Mixture_norm", u, 3, binary);
      write_array(o, "gradRho", grad_rho(c, rho), 1, binary);
    } else {
      for (int k = 0; k < np; k++) {  // PhasePUEq scalars (src/Models/PUEq/PhasePUEq.cpp:60-110)
        std::string e = strip_xml(ecg_input_eos_name(in, k));
        std::vector<double> a = f[k], r = f[np + k], t = slice(T, k), y = slice(Y, k);
        for (int64_t i = 0; i < n; i++) {
          if (a[i] < 1.e-20) a[i] = 0.;
          if (r[i] < 1.e-20) r[i] = 1.e-20;
          if (t[i] < 1.e-20) t[i] = 1.e-20;
          if (y[i] < 1.e-20) y[i] = 0.;
        }
        write_array(o, "F" + std::to_string(k) + "_Alpha_" + e, a, 1, binary);
        write_array(o, "F" + std::to_string(k) + "_Density_" + e, r, 1, binary);
        write_array(o, "F" + std::to_string(k) + "_Temperature_" + e, t, 1, binary);
        write_array(o, "F" + std::to_string(k) + "_Mass fraction_" + e, y, 1, binary);
      }
      std::vector<double> rho((size_t)n, 0.);
      for (int k = 0; k < np; k++)
        for (int64_t i = 0; i < n; i++) rho[i] += f[k][i] * f[np + k][i];
      write_array(o, "Density_Mixture", rho, 1, binary);
      write_array(o, "Pressure_Mixture", f[2 * np], 1, binary);
      write_array(o, "Total_energy_Mixture", f[2 * np + 4], 1, binary);
      std::vector<double> u((size_t)3 * n);
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) u[3 * i + d] = f[2 * np + 1 + d][i];
      write_array(o, "Velocity_Mixture", u, 3, binary);
      write_transports(o, f, 2 * np + 5);
      write_array(o, "gradRho", grad_rho(c, rho), 1, binary);
    }
    o << "      </CellData>\n    </Piece>\n  </RectilinearGrid>\n</VTKFile>\n";
    return (bool)o;
  }
};

int run_case(const std::string& work, const std::string& rel) {
  std::string cdir = work + rel;
  ecg_input* in = nullptr;
  ecg_status s = ecg_input_read(cdir.c_str(), (work + "libEOS").c_str(), &in);
  if (s != ECG_OK) {
    std::fprintf(stderr, "%s: %s: %s\n", rel.c_str(), ecg_status_str(s), ecg_last_error());
    return 1;
  }
  ecg_case c;
  ecg_input_case(in, &c);
  int32_t iter_freq = 0;
  double time_freq = 0.;
  ecg_input_print_control(in, &iter_freq, &time_freq);
  const int64_t n = (int64_t)c.ncells[0] * c.ncells[1] * c.ncells[2];
  ecg_ctx* ctx = nullptr;
  s = ecg_create(&c, &ctx);
  if (s != ECG_OK) {
    std::fprintf(stderr, "%s: %s: %s\n", rel.c_str(), ecg_status_str(s), ecg_last_error());
    ecg_input_free(in);
    return 1;
  }
  int32_t binary = 1, precision = 0, restart = 0;
  ecg_input_output_control(in, &binary, &precision, &restart);
  const int nf = abi_fields(c);
  std::vector<std::vector<double>> f(nf, std::vector<double>((size_t)n));
  std::vector<double*> ptr;
  for (auto& v : f) ptr.push_back(v.data());
  std::string out = work + "results/" + ecg_input_run_name(in) + "/";
  Output w{out, in, c, n, 0, binary != 0, precision};
  double dt = 1.e-15, t = 0.;
  int32_t it = 0;
  std::string fail_msg;
  // infoCalcul.out lines as Output::saveInfos writes them (src/InputOutput/Output.cpp:491-515): the CPU
  // count, then "file iteration time nextDt computeSeconds amrSeconds commSeconds" per print
  std::vector<std::string> info_lines;
  if (restart > 0) {
    // Output::readInfos :524: the line of file N gives iteration, time and the next dt (as printed)
    std::ifstream fi(out + "infoCalcul.out");
    std::string line;
    bool found = false;
    if (fi && std::getline(fi, line)) {
      info_lines.push_back(line);
      if (std::atoi(line.c_str()) != 1) fail_msg = "restart needs a single-CPU infoCalcul.out";
      while (fail_msg.empty() && std::getline(fi, line)) {
        info_lines.push_back(line);
        std::istringstream ls(line);
        int num = -1;
        ls >> num;
        if (num == restart) {
          ls >> it >> t >> dt;
          found = (bool)ls;
          break;
        }
      }
    }
    if (fail_msg.empty() && !found) fail_msg = "restart not possible - check file 'infoCalcul.out'";
    std::vector<std::vector<double>> arrays;
    if (fail_msg.empty() && !read_cell_arrays(out + "datasets/" + result_name(binary != 0, restart), arrays, &fail_msg))
      fail_msg = "restart: " + fail_msg;
    if (fail_msg.empty()) {
      // phase scalars then vectors, mixture scalars then vectors (OutputXML::ReadPhysicalDataXML :194)
      const int np = c.nphases;
      const bool euler = c.model == ECG_MODEL_EULER;
      const bool ptueq = c.model == ECG_MODEL_PTUEQ;
      const size_t base = euler ? 4 : (ptueq ? (size_t)2 * np + 4 : (size_t)4 * np + 4);
      const size_t need = base + c.ntransports;  // then the transports T1, T2, ...
      bool ok = arrays.size() >= need;
      for (size_t a = 0; ok && a < need; a++) {
        bool vec = euler ? a == 3 : a == base - 1;
        ok = arrays[a].size() == (size_t)n * (vec ? 3 : 1);
      }
      if (!ok) {
        fail_msg = "restart: result file does not hold this case's fields";
      } else if (ptueq) {  // F<k> alpha, density; mixture density, pressure, temperature, velocity
        for (int k = 0; k < np; k++) {
          f[k] = arrays[2 * k];
          f[np + k] = arrays[2 * k + 1];
        }
        f[2 * np] = arrays[2 * np + 1];
        f[2 * np + 5] = arrays[2 * np + 2];
        for (int64_t i = 0; i < n; i++)
          for (int d = 0; d < 3; d++) f[2 * np + 1 + d][i] = arrays[2 * np + 3][3 * i + d];
      } else if (euler) {  // F0 density, pressure, temperature, velocity
        f[0] = arrays[0];
        f[1] = arrays[1];
        for (int64_t i = 0; i < n; i++)
          for (int d = 0; d < 3; d++) f[2 + d][i] = arrays[3][3 * i + d];
      } else {  // F<k> alpha, density, temperature, mass fraction; mixture density, pressure, energy, velocity
        for (int k = 0; k < np; k++) {
          f[k] = arrays[4 * k];
          f[np + k] = arrays[4 * k + 1];
        }
        f[2 * np] = arrays[4 * np + 1];
        f[2 * np + 4] = arrays[4 * np + 2];
        for (int64_t i = 0; i < n; i++)
          for (int d = 0; d < 3; d++) f[2 * np + 1 + d][i] = arrays[4 * np + 3][3 * i + d];
      }
      if (ok) {
        const int first = euler ? 6 : 2 * np + 5;
        for (int j = 0; j < c.ntransports; j++) f[first + j] = arrays[base + j];
      }
    }
    if (fail_msg.empty()) {
      s = ecg_restart_fill(&c, ptr.data(), n);
      if (s == ECG_OK) s = ecg_upload_prim(ctx, ptr.data(), n);
      if (s != ECG_OK) fail_msg = ecg_last_error();
    }
    w.file = restart + 1;
  } else {
    s = ecg_input_fill(in, ptr.data(), n);
    if (s == ECG_OK) s = ecg_upload_prim(ctx, ptr.data(), n);
    if (s != ECG_OK) fail_msg = ecg_last_error();
  }
  if (fail_msg.empty() && !mkdirs(out + "datasets")) fail_msg = "cannot create " + out + "datasets";
  if (!fail_msg.empty()) {
    std::fprintf(stderr, "%s: cannot start: %s\n", rel.c_str(), fail_msg.c_str());
    ecg_destroy(ctx);
    ecg_input_free(in);
    return 1;
  }
  std::ofstream info(out + "infoCalcul.out", std::ios::trunc);
  if (precision != 0) info.precision(precision);
  const std::clock_t clock0 = std::clock();
  auto save_info = [&](double next_dt) {
    double secs = (double)(std::clock() - clock0) / CLOCKS_PER_SEC;
    info << w.file - 1 << " " << it << " " << t << " " << next_dt << " " << secs << " " << 0. << " " << 0. << std::endl;
  };
  if (restart > 0) {
    for (auto& l : info_lines) info << l << std::endl;
  } else {
    info << 1 << std::endl;
    w.write(ctx);
    save_info(0.);  // the next dt is not known before the first step (printed as 0)
  }
  std::printf("T | %s: %lld cells, %s%s\n", rel.c_str(), (long long)n, c.time_iterations ? "iterations" : "physical time",
              restart > 0 ? ", restarted" : "");
  double next_print = t + time_freq;
  int rc = 0;
  for (bool finished = false; !finished;) {
    int32_t chunk = 1;
    if (c.time_iterations) {  // steps up to the next print in one call
      int32_t to_print = iter_freq > 0 ? iter_freq - (it % iter_freq) : c.max_iterations - it;
      chunk = std::min(to_print, c.max_iterations - it);
      if (chunk < 1) chunk = 1;
    }
    ecg_step_stats st;
    s = ecg_step(ctx, chunk, &dt, &t, &st);
    if (s != ECG_OK) {
      std::fprintf(stderr, "%s: %s: %s\n", rel.c_str(), ecg_status_str(s), ecg_last_error());
      rc = 1;
      break;
    }
    it += chunk;
    bool print = false;
    if (c.time_iterations) {
      if (iter_freq > 0 && it % iter_freq == 0) print = true;
      if (it >= c.max_iterations) finished = true;
    } else {
      if (t >= next_print) {
        print = true;
        next_print += time_freq;
      }
      if (t >= c.total_time) {
        print = true;
        finished = true;
      }
    }
    if (print) {
      w.write(ctx);
      save_info(dt);
      std::printf("T | iteration %d, t = %.6e s, dt = %.6e s, file %d\n", it, t, dt, w.file - 1);
    }
  }
  ecg_destroy(ctx);
  ecg_input_free(in);
  return rc;
}

}  // namespace

int main(int argc, char** argv) {
  std::string work = argc > 1 ? argv[1] : "./";
  if (work.back() != '/') work += '/';
  std::ifstream f(work + "ECOGEN.xml");
  if (!f) {
    std::fprintf(stderr, "cannot open %sECOGEN.xml\n", work.c_str());
    return 1;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string txt = ss.str();
  // <testCase>folder/</testCase> entries outside comments (src/main.cpp:82)
  std::vector<std::string> cases;
  size_t pos = 0;
  while (true) {
    size_t c0 = txt.find("<!--", pos), t0 = txt.find("<testCase>", pos);
    if (t0 == std::string::npos) break;
    if (c0 != std::string::npos && c0 < t0) {
      size_t c1 = txt.find("-->", c0);
      if (c1 == std::string::npos) break;
      pos = c1 + 3;
      continue;
    }
    size_t t1 = txt.find("</testCase>", t0);
    if (t1 == std::string::npos) break;
    std::string name = txt.substr(t0 + 10, t1 - t0 - 10);
    size_t a = name.find_first_not_of(" \t\r\n"), b = name.find_last_not_of(" \t\r\n");
    if (a != std::string::npos) cases.push_back(name.substr(a, b - a + 1));
    pos = t1 + 11;
  }
  int failed = 0;
  for (auto& c : cases) failed += run_case(work, c);
  return failed;
}
