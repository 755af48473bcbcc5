// ecogen-b200: command-line driver with ECOGEN's interface, built on the C ABI.
//
//   ecogen-b200 <work folder>
//
// Like the reference's main (src/main.cpp:44-133) it reads <work>/ECOGEN.xml, runs each <testCase>
// folder in turn with the EOS files of <work>/libEOS, and writes results to
// <work>/results/<run>/: infoCalcul.out (iteration, time, dt per print) and, at every print time,
// datasets/resultB64_CPU0_TIME<k>.vtr — a VTK rectilinear grid with base64 Float64 cell arrays named
// like the reference's writer (src/InputOutput/OutputXML.cpp:320-470).  Print control follows
// Run::solver (src/Run.cpp:417-428): every iterFreq iterations, or every timeFreq of physical time
// and at the end.  A case the library does not run is reported and skipped; the exit code is the
// number of failed cases.
#include <sys/stat.h>

#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

extern "C" {
#include "../../include/ecogen_b200.h"
}

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

// VTK "binary" inline array: base64 of a 4-byte length header, then base64 of the data
void write_array(std::ostream& f, const std::string& name, const std::vector<double>& v, int ncomp) {
  f << "        <DataArray type=\"Float64\"";
  if (!name.empty()) f << " Name=\"" << name << "\"";
  if (ncomp > 1) f << " NumberOfComponents=\"" << ncomp << "\"";
  f << " format=\"binary\">\n";
  int32_t nb = (int32_t)(v.size() * sizeof(double));
  f << b64(reinterpret_cast<const unsigned char*>(&nb), 4)
    << b64(reinterpret_cast<const unsigned char*>(v.data()), v.size() * sizeof(double)) << "\n";
  f << "        </DataArray>\n";
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

struct Output {
  std::string dir;
  const ecg_input* in;
  ecg_case c;
  int64_t n;
  int file = 0;

  bool write(ecg_ctx* ctx) {
    const int np = c.nphases;
    const bool euler = c.model == ECG_MODEL_EULER;
    const int nf = euler ? 6 : 2 * np + 5;
    std::vector<std::vector<double>> f(nf, std::vector<double>((size_t)n));
    std::vector<double*> ptr;
    for (auto& v : f) ptr.push_back(v.data());
    if (ecg_download_prim(ctx, ptr.data(), n) != ECG_OK) return false;
    std::vector<double> T((size_t)np * n), Y((size_t)np * n);
    if (ecg_download_derived(ctx, T.data(), Y.data(), n) != ECG_OK) return false;
    char name[64];
    std::snprintf(name, sizeof(name), "resultB64_CPU0_TIME%d.vtr", file++);
    std::ofstream o(dir + "datasets/" + name, std::ios::trunc);
    if (!o) return false;
    int nx = c.ncells[0], ny = c.ncells[1], nz = c.ncells[2];
    o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"RectilinearGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n";
    o << "  <RectilinearGrid WholeExtent=\"0 " << nx << " 0 " << ny << " 0 " << nz << "\">\n";
    o << "    <Piece Extent=\"0 " << nx << " 0 " << ny << " 0 " << nz << "\">\n      <Coordinates>\n";
    for (int a = 0; a < 3; a++) {
      std::vector<double> x((size_t)c.ncells[a] + 1);
      double d = c.length[a] / (double)c.ncells[a];
      for (int i = 0; i <= c.ncells[a]; i++) x[i] = i * d;
      write_array(o, "", x, 1);
    }
    o << "      </Coordinates>\n      <CellData>\n";
    auto slice = [&](const std::vector<double>& v, int k) {
      return std::vector<double>(v.begin() + (size_t)k * n, v.begin() + (size_t)(k + 1) * n);
    };
    if (euler) {
      std::string e = strip_xml(ecg_input_eos_name(in, 0));
      write_array(o, "F0_Density_" + e, f[0], 1);
      write_array(o, "F0_Pressure_" + e, f[1], 1);
      write_array(o, "F0_Temperature_" + e, slice(T, 0), 1);
      std::vector<double> u((size_t)3 * n);
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) u[3 * i + d] = f[2 + d][i];
      write_array(o, "F0_Velocity_" + e, u, 3);
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
        write_array(o, "F" + std::to_string(k) + "_Alpha_" + e, a, 1);
        write_array(o, "F" + std::to_string(k) + "_Density_" + e, r, 1);
        write_array(o, "F" + std::to_string(k) + "_Temperature_" + e, t, 1);
        write_array(o, "F" + std::to_string(k) + "_Mass fraction_" + e, y, 1);
      }
      std::vector<double> rho((size_t)n, 0.);
      for (int k = 0; k < np; k++)
        for (int64_t i = 0; i < n; i++) rho[i] += f[k][i] * f[np + k][i];
      write_array(o, "Density_Mixture", rho, 1);
      write_array(o, "Pressure_Mixture", f[2 * np], 1);
      write_array(o, "Total_energy_Mixture", f[2 * np + 4], 1);
      std::vector<double> u((size_t)3 * n);
      for (int64_t i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) u[3 * i + d] = f[2 * np + 1 + d][i];
      write_array(o, "Velocity_Mixture", u, 3);
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
  const int nf = c.model == ECG_MODEL_EULER ? 6 : 2 * c.nphases + 5;
  std::vector<std::vector<double>> f(nf, std::vector<double>((size_t)n));
  std::vector<double*> ptr;
  for (auto& v : f) ptr.push_back(v.data());
  s = ecg_input_fill(in, ptr.data(), n);
  if (s == ECG_OK) s = ecg_upload_prim(ctx, ptr.data(), n);
  std::string out = work + "results/" + ecg_input_run_name(in) + "/";
  if (s != ECG_OK || !mkdirs(out + "datasets")) {
    std::fprintf(stderr, "%s: cannot start: %s\n", rel.c_str(), ecg_last_error());
    ecg_destroy(ctx);
    ecg_input_free(in);
    return 1;
  }
  Output w{out, in, c, n, 0};
  std::ofstream info(out + "infoCalcul.out", std::ios::trunc);
  info.precision(17);
  double dt = 1.e-15, t = 0.;
  int32_t it = 0;
  w.write(ctx);
  info << w.file - 1 << " " << it << " " << t << " " << dt << "\n";
  std::printf("T | %s: %lld cells, %s\n", rel.c_str(), (long long)n, c.time_iterations ? "iterations" : "physical time");
  double next_print = time_freq;
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
      info << w.file - 1 << " " << it << " " << t << " " << dt << "\n";
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
