// Case input: the four ECOGEN XML files of a case plus its EOS files, and the initial
// condition fill.  Restates, for the Cartesian Euler / Kapila cases this library runs,
// Input::inputMain / inputMesh / inputModel / inputEOS / inputInitialConditions
// (src/InputOutput/Input.cpp:77, :319, :566, :865, :917), the geometric domains of
// src/Geometries/ and Cell::completeFulfillState (src/Order1/Cell.cpp:344).
// Inputs this library does not run are refused with ECG_ERR_UNSUPPORTED instead of being
// silently ignored.
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ecogen_b200.h"
#include "ecg_internal.h"
#include "ecg_xml.h"

using ecg::xml::Node;
using ecg::xml::upper;

struct Domain {
  int kind;  // 0 entire, 1 halfSpace, 2 disc, 3 sphere, 4 rectangle, 5 cuboid
  int axis = 0, axis1 = 0, axis2 = 0, direction = 1;
  double origin = 0., radius = 0., l1 = 0., l2 = 0., lx = 0., ly = 0., lz = 0.;
  double c[3] = {0., 0., 0.};
  int state = -1;
};

struct StateIC {
  std::string name;
  double alpha[ECG_MAX_PHASES], rho[ECG_MAX_PHASES];
  double p = 0.;
  double T = 0.;            // mixture temperature (temperature-pressure equilibrium model)
  double u[3] = {0., 0., 0.};
  double tr[2] = {0., 0.};  // passive transports (0 unless the state gives them)
};

struct ecg_input {
  ecg_case c;
  int iter_freq = 0;
  double time_freq = 0.;
  int binary = 1, precision = 0, restart_file = 0;
  std::string run_name;
  std::string output_format;
  std::vector<std::string> eos_names;
  std::vector<std::string> transport_names;
  std::vector<StateIC> states;
  std::vector<Domain> domains;
};

namespace {

ecg_status fail(ecg_status s, const std::string& msg) {
  ecg::set_error(msg);
  return s;
}

int axis_of(const std::string& a) {
  std::string u = upper(a);
  if (u == "X") return 0;
  if (u == "Y") return 1;
  if (u == "Z") return 2;
  return -1;
}

// EOS helpers used by the initial fill (same formulas as the reference EOS classes).
double eos_density_pT(const ecg_eos& q, double eps, double p, double T) {  // computeDensity
  if (q.type == ECG_EOS_IG) return p / std::max((q.gamma - 1.) * q.cv * T, eps);
  if (q.type == ECG_EOS_SG) return (p + q.pinf) / std::max((q.gamma - 1.) * q.cv * T, eps);
  return (p + q.pinf) / std::max((q.gamma - 1.) * q.cv * T + q.b * (p + q.pinf), eps);
}

// Total energy of a temperature-pressure equilibrium cell from the ABI fields alpha_k (0, 1), rho_k (2, 3),
// p (4), u (5-7): ModPTUEq::fulfillState (e_k), MixPTUEq::computeMixtureVariables (e = sum Y_k e_k) and
// computeTotalEnergy (E = e + |u|^2 / 2).
double ptueq_total_energy(const ecg_case& c, double* const* f, int64_t i) {
  double rho = 0., e = 0., ek[2];
  for (int k = 0; k < 2; k++) {
    ek[k] = ecg::host_eos_e(c.eos[k], 0., f[2 + k][i], f[4][i]);
    rho += f[k][i] * f[2 + k][i];
  }
  for (int k = 0; k < 2; k++) e += f[k][i] * f[2 + k][i] / rho * ek[k];
  const double u0 = f[5][i], u1 = f[6][i], u2 = f[7][i];
  return e + 0.5 * (u0 * u0 + u1 * u1 + u2 * u2);
}

ecg_status read_eos(const std::string& dir, const std::string& name, ecg_eos* e) {
  std::string err;
  std::string path = dir + "/" + name;
  auto root = ecg::xml::parse_file(path, &err);
  if (!root) return fail(ECG_ERR_XML, err);
  if (root->name != "parametersEOS") return fail(ECG_ERR_XML, path + ": root parametersEOS expected");
  const Node* t = root->child("EOS");
  if (!t || !t->has("type")) return fail(ECG_ERR_XML, path + ": <EOS type> missing");
  std::string type = upper(t->attr("type"));
  const Node* pr = root->child("parameters");
  if (!pr) return fail(ECG_ERR_XML, path + ": <parameters> missing");
  std::memset(e, 0, sizeof(*e));
  std::vector<std::pair<const char*, double*>> want;
  if (type == "IG") {
    e->type = ECG_EOS_IG;
    want = {{"gamma", &e->gamma}, {"cv", &e->cv}, {"energyRef", &e->eref}, {"entropyRef", &e->sref}};
  } else if (type == "SG") {
    e->type = ECG_EOS_SG;
    want = {{"gamma", &e->gamma}, {"pInf", &e->pinf}, {"cv", &e->cv}, {"energyRef", &e->eref}, {"entropyRef", &e->sref}};
  } else if (type == "NASG") {
    e->type = ECG_EOS_NASG;
    want = {{"gamma", &e->gamma}, {"pInf", &e->pinf}, {"b", &e->b},
            {"cv", &e->cv},       {"energyRef", &e->eref}, {"entropyRef", &e->sref}};
  } else {
    return fail(ECG_ERR_UNSUPPORTED, path + ": EOS type " + type + " is not supported (IG, SG, NASG)");
  }
  for (auto& w : want)
    if (!pr->get_double(w.first, w.second)) return fail(ECG_ERR_XML, path + ": attribute " + w.first + " missing");
  return ECG_OK;
}

int limiter_code(const std::string& s) {
  std::string u = upper(ecg::xml::trim(s));
  if (u == "MINMOD") return ECG_LIM_MINMOD;
  if (u == "VANLEER") return ECG_LIM_VANLEER;
  if (u == "VANALBADA") return ECG_LIM_VANALBADA;
  if (u == "SUPERBEE") return ECG_LIM_SUPERBEE;
  if (u == "MC") return ECG_LIM_MC;
  if (u == "THINC") return ECG_LIM_THINC;
  return -1;
}

}  // namespace

extern "C" ecg_status ecg_input_read(const char* case_dir, const char* eos_dir, ecg_input** out) {
  if (!case_dir || !eos_dir || !out) return fail(ECG_ERR_INVALID, "ecg_input_read: null argument");
  *out = nullptr;
  auto in = new ecg_input();
  std::memset(&in->c, 0, sizeof(in->c));
  ecg_case& c = in->c;
  std::string dir(case_dir);
  if (!dir.empty() && dir.back() != '/') dir += '/';
  std::string err;
  auto bail = [&](ecg_status s, const std::string& m) {
    delete in;
    return fail(s, m);
  };

  // ---------------------------------------------------------------- main.xml (Input::inputMain :77)
  auto mainx = ecg::xml::parse_file(dir + "main.xml", &err);
  if (!mainx) return bail(ECG_ERR_XML, err);
  if (mainx->name != "computationParam") return bail(ECG_ERR_XML, "main.xml: root computationParam expected");
  const Node* run = mainx->child("run");
  if (!run || ecg::xml::trim(run->text).empty()) return bail(ECG_ERR_XML, "main.xml: <run> missing");
  in->run_name = ecg::xml::trim(run->text);
  const Node* om = mainx->child("outputMode");
  if (!om || om->attr("format").empty()) return bail(ECG_ERR_XML, "main.xml: <outputMode format> missing");
  in->output_format = upper(om->attr("format"));
  {  // Output::Output src/InputOutput/Output.cpp:73-80: precision optional, binary required
    bool bin = true;
    if (!om->get_bool("binary", &bin)) return bail(ECG_ERR_XML, "main.xml: <outputMode binary> missing");
    in->binary = bin ? 1 : 0;
    int prec = 0;
    if (om->get_int("precision", &prec)) in->precision = prec;
  }
  const Node* tc = mainx->child("timeControlMode");
  bool iters = false;
  if (!tc || !tc->get_bool("iterations", &iters)) return bail(ECG_ERR_XML, "main.xml: <timeControlMode iterations> missing");
  c.time_iterations = iters ? 1 : 0;
  if (iters) {
    const Node* it = tc->child("iterations");
    int nb = 0;
    if (!it || !it->get_int("number", &nb)) return bail(ECG_ERR_XML, "main.xml: <iterations number> missing");
    if (!it->get_int("iterFreq", &in->iter_freq)) return bail(ECG_ERR_XML, "main.xml: <iterations iterFreq> missing");
    c.max_iterations = nb;
  } else {
    const Node* pt = tc->child("physicalTime");
    if (!pt || !pt->get_double("totalTime", &c.total_time)) return bail(ECG_ERR_XML, "main.xml: <physicalTime totalTime> missing");
    if (!pt->get_double("timeFreq", &in->time_freq)) return bail(ECG_ERR_XML, "main.xml: <physicalTime timeFreq> missing");
  }
  const Node* cc = mainx->child("computationControl");
  if (!cc || !cc->get_double("CFL", &c.cfl)) return bail(ECG_ERR_XML, "main.xml: <computationControl CFL> missing");
  const Node* so = mainx->child("secondOrder");
  if (!so) {
    c.order = 1;
    for (int i = 0; i < 4; i++) c.limiter[i] = ECG_LIM_NONE;
  } else {
    c.order = 2;
    const Node* g = so->child("globalLimiter");
    if (!g) return bail(ECG_ERR_XML, "main.xml: <globalLimiter> missing");
    int gl = limiter_code(g->text);
    if (gl < 0) return bail(ECG_ERR_XML, "main.xml: unknown global limiter");
    if (gl == ECG_LIM_THINC) return bail(ECG_ERR_XML, "THINC can only be a volume-fraction limiter");
    int il = gl;
    if (const Node* n = so->child("interfaceLimiter")) il = limiter_code(n->text);
    if (il < 0 || il == ECG_LIM_THINC) return bail(ECG_ERR_XML, "main.xml: bad interface limiter");
    int gv = gl;
    if (const Node* n = so->child("globalVolumeFractionLimiter")) gv = limiter_code(n->text);
    int iv = il;
    if (const Node* n = so->child("interfaceVolumeFractionLimiter")) iv = limiter_code(n->text);
    if (gv < 0 || iv < 0) return bail(ECG_ERR_XML, "main.xml: bad volume-fraction limiter");
    c.limiter[0] = gl;
    c.limiter[1] = il;
    c.limiter[2] = gv;
    c.limiter[3] = iv;
  }
  if (const Node* rs = mainx->child("restartSimulation")) {  // Input::inputMain :305-311
    int rn = 0, freq = 0;
    if (!rs->get_int("restartFileNumber", &rn)) return bail(ECG_ERR_XML, "main.xml: <restartSimulation restartFileNumber> missing");
    if (!rs->get_int("AMRsaveFreq", &freq)) return bail(ECG_ERR_XML, "main.xml: <restartSimulation AMRsaveFreq> missing");
    if (rn < 0) return bail(ECG_ERR_XML, "main.xml: negative restartFileNumber");
    in->restart_file = rn;
  }

  // ---------------------------------------------------------------- mesh.xml (Input::inputMesh :319)
  auto meshx = ecg::xml::parse_file(dir + "mesh.xml", &err);
  if (!meshx) return bail(ECG_ERR_XML, err);
  if (meshx->name != "mesh") return bail(ECG_ERR_XML, "mesh.xml: root mesh expected");
  const Node* ty = meshx->child("type");
  if (!ty || ty->attr("structure").empty()) return bail(ECG_ERR_XML, "mesh.xml: <type structure> missing");
  if (upper(ty->attr("structure")) != "CARTESIAN") return bail(ECG_ERR_UNSUPPORTED, "only Cartesian meshes are supported");
  const Node* cm = meshx->child("cartesianMesh");
  if (!cm) return bail(ECG_ERR_XML, "mesh.xml: <cartesianMesh> missing");
  const Node* dm = cm->child("dimensions");
  if (!dm || !dm->get_double("x", &c.length[0]) || !dm->get_double("y", &c.length[1]) || !dm->get_double("z", &c.length[2]))
    return bail(ECG_ERR_XML, "mesh.xml: <dimensions x y z> missing");
  const Node* nc = cm->child("numberCells");
  if (!nc || !nc->get_int("x", &c.ncells[0]) || !nc->get_int("y", &c.ncells[1]) || !nc->get_int("z", &c.ncells[2]))
    return bail(ECG_ERR_XML, "mesh.xml: <numberCells x y z> missing");
  if (c.ncells[0] <= 1) return bail(ECG_ERR_XML, "Number of cells in the x-direction has to be superior to 1");
  if (c.ncells[2] > 1 && c.ncells[1] <= 1)
    return bail(ECG_ERR_XML, "Number of cells in the z-direction can't be superior to 1 if number of cells in the y-direction is equal to 1");
  if (const Node* ms = cm->child("meshStretching")) {
    // Input::inputMesh src/InputOutput/Input.cpp:460-520: zones per axis with more than one cell, checked
    // like stretchZone::verifyStretching (src/Meshes/stretchZone.cpp:74-93); the axis then has the sum of
    // its zones' cells (MeshCartesian::meshStretching src/Meshes/MeshCartesian.cpp:168-210)
    const char* tags[3] = {"XStretching", "YStretching", "ZStretching"};
    for (int a = 0; a < 3; a++) {
      if (c.ncells[a] <= 1) continue;
      const Node* ax = ms->child(tags[a]);
      if (!ax) continue;
      int nz = 0, cells = 0;
      for (const Node* st : ax->all("stretch")) {
        if (nz == ECG_MAX_STRETCH_ZONES) return bail(ECG_ERR_UNSUPPORTED, "more than 8 stretch zones on an axis");
        ecg_stretch_zone& z = c.stretch[a][nz];
        if (!st->get_double("startAt", &z.start)) return bail(ECG_ERR_XML, "mesh.xml: <stretch startAt> missing");
        if (!st->get_double("endAt", &z.end)) return bail(ECG_ERR_XML, "mesh.xml: <stretch endAt> missing");
        if (!st->get_double("factor", &z.factor)) return bail(ECG_ERR_XML, "mesh.xml: <stretch factor> missing");
        if (!st->get_int("numberCells", &z.ncells)) return bail(ECG_ERR_XML, "mesh.xml: <stretch numberCells> missing");
        if (z.ncells < 1) return bail(ECG_ERR_XML, "mesh.xml: <stretch numberCells> below 1");
        cells += z.ncells;
        nz++;
      }
      if (nz == 0) continue;
      const bool ok_start = c.stretch[a][0].start == 0., ok_end = c.stretch[a][nz - 1].end == c.length[a];
      bool contiguous = true;
      for (int z = 1; z < nz; z++) contiguous = contiguous && c.stretch[a][z].start == c.stretch[a][z - 1].end;
      if (!ok_start || !ok_end || !contiguous) return bail(ECG_ERR_XML, "mesh.xml: stretching zones (ErrorXMLStretching)");
      c.nstretch[a] = nz;
      c.ncells[a] = cells;
    }
  }
  if (cm->child("AMR")) return bail(ECG_ERR_UNSUPPORTED, "AMR is not supported");

  // ---------------------------------------------------------------- model.xml (Input::inputModel :566)
  auto modx = ecg::xml::parse_file(dir + "model.xml", &err);
  if (!modx) return bail(ECG_ERR_XML, err);
  if (modx->name != "model") return bail(ECG_ERR_XML, "model.xml: root model expected");
  const Node* fm = modx->child("flowModel");
  if (!fm || fm->attr("name").empty()) return bail(ECG_ERR_XML, "model.xml: <flowModel name> missing");
  std::string model = upper(fm->attr("name"));
  int ntr = 0;
  fm->get_int("numberTransports", &ntr);
  if (ntr < 0) return bail(ECG_ERR_XML, "model.xml: negative numberTransports");
  if (ntr > 2) return bail(ECG_ERR_UNSUPPORTED, "more than two passive transports are not supported");
  c.ntransports = ntr;
  {  // Input::inputModel src/InputOutput/Input.cpp:707-719: names in order, at least numberTransports
    std::vector<std::string> names;
    for (const Node* t : modx->all("transport")) {
      if (t->attr("name").empty()) return bail(ECG_ERR_XML, "model.xml: <transport name> missing");
      names.push_back(t->attr("name"));
    }
    if ((int)names.size() < ntr) return bail(ECG_ERR_XML, "model.xml: fewer <transport> than numberTransports");
    in->transport_names = names;
  }
  bool alpha_null = false;
  if (model == "EULER") {
    c.model = ECG_MODEL_EULER;
    c.nphases = 1;
  } else if (model == "PRESSUREVELOCITYEQ") {
    c.model = ECG_MODEL_KAPILA;
    if (!fm->get_int("numberPhases", &c.nphases)) return bail(ECG_ERR_XML, "model.xml: numberPhases missing");
    if (!fm->get_bool("alphaNull", &alpha_null)) return bail(ECG_ERR_XML, "model.xml: alphaNull missing");
    if (c.nphases < 2 || c.nphases > ECG_MAX_PHASES)
      return bail(ECG_ERR_UNSUPPORTED, "Kapila runs need 2 or 3 phases");
  } else if (model == "TEMPERATUREPRESSUREVELOCITYEQ") {  // Input.cpp:642, ModPTUEq (no alphaNull attribute)
    c.model = ECG_MODEL_PTUEQ;
    if (!fm->get_int("numberPhases", &c.nphases)) return bail(ECG_ERR_XML, "model.xml: numberPhases missing");
    if (c.nphases != 2)
      return bail(ECG_ERR_UNSUPPORTED, "more than two phases not permitted in thermal equilibrium model");
  } else {
    return bail(ECG_ERR_UNSUPPORTED, "flow model " + model +
                                         " is not supported (Euler, PressureVelocityEq, TemperaturePressureVelocityEq)");
  }
  c.alpha_null = alpha_null ? 1 : 0;
  if (const Node* lm = modx->child("lowMach")) {
    bool st = false;
    if (lm->get_bool("state", &st) && st) return bail(ECG_ERR_UNSUPPORTED, "low-Mach preconditioning is not supported");
  }
  for (const Node* e : modx->all("EOS")) {
    if (e->attr("name").empty()) return bail(ECG_ERR_XML, "model.xml: <EOS name> missing");
    in->eos_names.push_back(e->attr("name"));
  }
  if ((int)in->eos_names.size() != c.nphases) return bail(ECG_ERR_XML, "model.xml: one EOS per phase expected");
  for (int k = 0; k < c.nphases; k++) {
    ecg_status s = read_eos(eos_dir, in->eos_names[k], &c.eos[k]);
    if (s != ECG_OK) {
      delete in;
      return s;
    }
  }
  if (modx->child("additionalPhysic")) return bail(ECG_ERR_UNSUPPORTED, "additional physics are not supported");
  if (modx->child("symmetryTerm")) return bail(ECG_ERR_UNSUPPORTED, "symmetry terms are not supported");
  if (modx->child("sourceTerms")) return bail(ECG_ERR_UNSUPPORTED, "source terms are not supported");
  if (c.model == ECG_MODEL_PTUEQ) {
    for (int k = 0; k < c.nphases; k++)  // MixPTUEq::computePressure (:97-99)
      if (c.eos[k].type == ECG_EOS_NASG)
        return bail(ECG_ERR_UNSUPPORTED, "Only IG and SG permitted in thermal equilibrium model");
    if (ntr > 0)  // no transport Riemann solver (src/Models/Model.h:185)
      return bail(ECG_ERR_UNSUPPORTED, "passive transports are not available for the thermal equilibrium model");
    if (modx->child("relaxation")) return bail(ECG_ERR_UNSUPPORTED, "relaxations of the thermal equilibrium model");
  }
  for (const Node* r : modx->all("relaxation")) {
    std::string t = upper(r->attr("type"));
    if (t == "PTMU") {
      if (c.ptmu) return bail(ECG_ERR_XML, "model.xml: PTMu relaxation given twice");
      if (c.model != ECG_MODEL_KAPILA || c.nphases != 2)
        return bail(ECG_ERR_XML, "Only two phases can be used with PTMu relaxation");
      const Node* d = r->child("dataPTMu");
      if (!d) return bail(ECG_ERR_XML, "model.xml: <dataPTMu> missing");
      std::string liq = d->attr("liquid"), vap = d->attr("vapor");
      c.ptmu = 1;
      c.ptmu_liquid = c.ptmu_vapor = -1;
      for (int k = 0; k < c.nphases; k++) {
        if (in->eos_names[k] == liq) c.ptmu_liquid = k;
        else if (in->eos_names[k] == vap) c.ptmu_vapor = k;
      }
      if (c.ptmu_liquid < 0 || c.ptmu_vapor < 0) return bail(ECG_ERR_XML, "model.xml: dataPTMu names no model EOS");
      for (int k = 0; k < 2; k++)
        if (c.eos[k].type == ECG_EOS_NASG) return bail(ECG_ERR_UNSUPPORTED, "PTMu saturation needs IG or SG phases");
    } else if (t == "PT") {  // RelaxationPT (Input.cpp:834-840), appended after the pressure relaxation
      if (c.pt_relaxation) return bail(ECG_ERR_XML, "model.xml: PT relaxation given twice");
      if (c.model != ECG_MODEL_KAPILA || c.nphases != 2)
        return bail(ECG_ERR_UNSUPPORTED, "PT relaxation is built for two phases");
      for (int k = 0; k < 2; k++)
        if (c.eos[k].type == ECG_EOS_NASG) return bail(ECG_ERR_UNSUPPORTED, "PT relaxation needs IG or SG phases");
      c.pt_relaxation = 1;
    } else if (t == "P") {
      std::string sp = upper(r->attr("speed"));
      if (sp == "FINITE") return bail(ECG_ERR_UNSUPPORTED, "finite-rate pressure relaxation is not supported");
    } else {
      return bail(ECG_ERR_UNSUPPORTED, "relaxation " + t + " is not supported");
    }
  }
  if (c.ptmu && c.pt_relaxation) return bail(ECG_ERR_UNSUPPORTED, "PTMu and PT relaxations together are not built");

  // ---------------------------------------------------------------- initialConditions.xml (:917)
  auto icx = ecg::xml::parse_file(dir + "initialConditions.xml", &err);
  if (!icx) return bail(ECG_ERR_XML, err);
  if (icx->name != "CI") return bail(ECG_ERR_XML, "initialConditions.xml: root CI expected");
  const Node* pd = icx->child("physicalDomains");
  if (!pd) return bail(ECG_ERR_XML, "initialConditions.xml: <physicalDomains> missing");
  double eps = c.alpha_null ? 1.e-15 : 0.;
  auto find_state = [&](const std::string& name) -> int {
    std::string un = upper(name);
    for (size_t i = 0; i < in->states.size(); i++)
      if (upper(in->states[i].name) == un) return (int)i;
    return -1;
  };
  for (const Node* d : pd->all("domain")) {
    std::string st = d->attr("state");
    if (d->attr("name").empty() || st.empty()) return bail(ECG_ERR_XML, "initialConditions.xml: domain name/state missing");
    int si = find_state(st);
    if (si < 0) {
      const Node* sn = nullptr;
      for (const Node* s : icx->all("state"))
        if (upper(s->attr("name")) == upper(st)) { sn = s; break; }
      if (!sn) return bail(ECG_ERR_XML, "initialConditions.xml: state " + st + " not found");
      StateIC S;
      S.name = sn->attr("name");
      int k = 0;
      if (c.model == ECG_MODEL_KAPILA || c.model == ECG_MODEL_PTUEQ) {
        const Node* mix = sn->child("mixture");
        const Node* dmx = mix ? mix->child("dataMix") : nullptr;
        const Node* vel = mix ? mix->child("velocity") : nullptr;
        if (!mix || !dmx || !dmx->get_double("pressure", &S.p)) return bail(ECG_ERR_XML, "state " + st + ": mixture pressure missing");
        // MixPTUEq::MixPTUEq src/Models/PTUEq/MixPTUEq.cpp:44-73: pressure and temperature
        if (c.model == ECG_MODEL_PTUEQ && !dmx->get_double("temperature", &S.T))
          return bail(ECG_ERR_XML, "state " + st + ": mixture temperature missing");
        if (!vel || !vel->get_double("x", &S.u[0]) || !vel->get_double("y", &S.u[1]) || !vel->get_double("z", &S.u[2]))
          return bail(ECG_ERR_XML, "state " + st + ": mixture velocity missing");
      }
      for (const Node* m : sn->all("material")) {
        if (k >= c.nphases) return bail(ECG_ERR_XML, "state " + st + ": too many materials");
        if (upper(m->attr("type")) != "FLUID") return bail(ECG_ERR_UNSUPPORTED, "only fluid materials are supported");
        if (m->attr("EOS") != in->eos_names[k])
          return bail(ECG_ERR_XML, "Materials in used states should be ordered in reference to model.xml");
        const Node* df = m->child("dataFluid");
        if (!df) return bail(ECG_ERR_XML, "state " + st + ": <dataFluid> missing");
        double rho = 0., T = 0., p = 0.;
        bool hr = df->get_double("density", &rho), hT = df->get_double("temperature", &T);
        if (c.model == ECG_MODEL_PTUEQ) {
          // PhasePTUEq::PhasePTUEq src/Models/PTUEq/PhasePTUEq.cpp:42-52: alpha only
          if (!df->get_double("alpha", &S.alpha[k])) return bail(ECG_ERR_XML, "state " + st + ": alpha missing");
          S.rho[k] = eos_density_pT(c.eos[k], 0., S.p, S.T);
        } else if (c.model == ECG_MODEL_KAPILA) {
          // PhasePUEq::PhasePUEq src/Models/PUEq/PhasePUEq.cpp:41-73
          if (!df->get_double("alpha", &S.alpha[k])) return bail(ECG_ERR_XML, "state " + st + ": alpha missing");
          if (hr && hT) return bail(ECG_ERR_XML, "only one of following is required : density, temperature");
          if (!hr && !hT) return bail(ECG_ERR_XML, "state " + st + ": density or temperature required");
          S.rho[k] = hT ? eos_density_pT(c.eos[k], eps, S.p, T) : rho;
        } else {
          // PhaseEuler::PhaseEuler src/Models/Euler/PhaseEuler.cpp:44-76
          bool hp = df->get_double("pressure", &p);
          if ((int)hr + (int)hp + (int)hT != 2) return bail(ECG_ERR_XML, "only two of following is required : density, pressure, temperature");
          if (hr && hT) return bail(ECG_ERR_XML, "impossible to initialize Euler phase with density and temperature");
          S.alpha[k] = 1.;
          S.rho[k] = hT ? eos_density_pT(c.eos[k], eps, p, T) : rho;
          S.p = p;
          const Node* vel = df->child("velocity");
          if (!vel || !vel->get_double("x", &S.u[0]) || !vel->get_double("y", &S.u[1]) || !vel->get_double("z", &S.u[2]))
            return bail(ECG_ERR_XML, "state " + st + ": velocity missing");
        }
        k++;
      }
      if (k != c.nphases) return bail(ECG_ERR_XML, "state " + st + ": one material per phase expected");
      {  // state transports (Input.cpp:1034-1050): matched by name, others ignored; a missing "value"
         // keeps the previous one read, as the reference's loop does
        double v = 0.;
        for (const Node* t : sn->all("transport")) {
          t->get_double("value", &v);
          for (int e = 0; e < c.ntransports; e++)
            if (t->attr("name") == in->transport_names[e]) {
              S.tr[e] = v;
              break;
            }
        }
      }
      in->states.push_back(S);
      si = (int)in->states.size() - 1;
    }
    Domain D;
    D.state = si;
    std::string type = upper(d->attr("type"));
    if (type == "ENTIREDOMAIN") {
      D.kind = 0;
    } else if (type == "HALFSPACE") {  // GDHalfSpace src/Geometries/GDHalfSpace.cpp:38-60
      const Node* h = d->child("dataHalfSpace");
      if (!h || !h->get_double("origin", &D.origin)) return bail(ECG_ERR_XML, "dataHalfSpace origin missing");
      D.kind = 1;
      D.axis = axis_of(h->attr("axis"));
      std::string dir2 = upper(h->attr("direction"));
      if (D.axis < 0) return bail(ECG_ERR_XML, "dataHalfSpace axis");
      if (dir2 == "POSITIVE") D.direction = 1;
      else if (dir2 == "NEGATIVE") D.direction = -1;
      else return bail(ECG_ERR_XML, "dataHalfSpace direction");
    } else if (type == "DISC") {  // GDDisc src/Geometries/GDDisc.cpp:38-70
      const Node* h = d->child("dataDisc");
      if (!h || !h->get_double("radius", &D.radius)) return bail(ECG_ERR_XML, "dataDisc radius missing");
      D.kind = 2;
      D.axis1 = axis_of(h->attr("axis1"));
      D.axis2 = axis_of(h->attr("axis2"));
      if (D.axis1 < 0 || D.axis2 < 0) return bail(ECG_ERR_XML, "dataDisc axes");
      const Node* ce = h->child("center");
      if (!ce) return bail(ECG_ERR_XML, "dataDisc center missing");
      ce->get_double("x", &D.c[0]);
      ce->get_double("y", &D.c[1]);
      ce->get_double("z", &D.c[2]);
    } else if (type == "SPHERE") {  // GDSphere src/Geometries/GDSphere.cpp:38-56
      const Node* h = d->child("dataSphere");
      if (!h || !h->get_double("radius", &D.radius)) return bail(ECG_ERR_XML, "dataSphere radius missing");
      D.kind = 3;
      const Node* ce = h->child("center");
      if (!ce) return bail(ECG_ERR_XML, "dataSphere center missing");
      ce->get_double("x", &D.c[0]);
      ce->get_double("y", &D.c[1]);
      ce->get_double("z", &D.c[2]);
    } else if (type == "RECTANGLE") {  // GDRectangle src/Geometries/GDRectangle.cpp:38-75
      const Node* h = d->child("dataRectangle");
      if (!h || !h->get_double("lAxis1", &D.l1) || !h->get_double("lAxis2", &D.l2))
        return bail(ECG_ERR_XML, "dataRectangle lengths missing");
      D.kind = 4;
      D.axis1 = axis_of(h->attr("axis1"));
      D.axis2 = axis_of(h->attr("axis2"));
      if (D.axis1 < 0 || D.axis2 < 0) return bail(ECG_ERR_XML, "dataRectangle axes");
      const Node* ce = h->child("posInferiorVertex");
      if (!ce) return bail(ECG_ERR_XML, "dataRectangle posInferiorVertex missing");
      ce->get_double("x", &D.c[0]);
      ce->get_double("y", &D.c[1]);
      ce->get_double("z", &D.c[2]);
    } else if (type == "CUBOID") {  // GDCuboid src/Geometries/GDCuboid.cpp:38-64
      const Node* h = d->child("dataCuboid");
      if (!h || !h->get_double("lAxisX", &D.lx) || !h->get_double("lAxisY", &D.ly) || !h->get_double("lAxisZ", &D.lz))
        return bail(ECG_ERR_XML, "dataCuboid lengths missing");
      D.kind = 5;
      const Node* ce = h->child("posInferiorVertex");
      if (!ce) return bail(ECG_ERR_XML, "dataCuboid posInferiorVertex missing");
      ce->get_double("x", &D.c[0]);
      ce->get_double("y", &D.c[1]);
      ce->get_double("z", &D.c[2]);
    } else {
      return bail(ECG_ERR_UNSUPPORTED, "domain type " + type + " is not supported");
    }
    in->domains.push_back(D);
  }
  if (in->domains.empty()) return bail(ECG_ERR_XML, "initialConditions.xml: no domain");
  const Node* bcs = icx->child("boundaryConditions");
  if (!bcs) return bail(ECG_ERR_XML, "initialConditions.xml: <boundaryConditions> missing");
  // The i-th <boundCond> in reading order is side i (Xm, Xp, Ym, Yp, Zm, Zp), whatever its "number"
  // (Input::readInputXML src/InputOutput/Input.cpp:1120-1190, MeshCartesian::assignLimits
  // src/Meshes/MeshCartesian.cpp:86); sides without one are non-reflecting.  Without viscosity
  // (out of scope here) a "wall" is a symmetry side.
  int side = 0;
  for (const Node* b : bcs->all("boundCond")) {
    int num = 0;
    if (b->attr("name").empty() || b->attr("type").empty() || !b->get_int("number", &num))
      return bail(ECG_ERR_XML, "boundCond name/type/number missing");
    if (side >= 6) return bail(ECG_ERR_XML, "more than six boundCond");
    std::string t = upper(b->attr("type"));
    if (t == "NONREFLECTING") in->c.bc[side] = ECG_BC_NONREFLECTING;
    else if (t == "SYMMETRY" || t == "WALL") in->c.bc[side] = ECG_BC_SYMMETRY;
    else
      return bail(ECG_ERR_UNSUPPORTED,
                  "boundary condition " + b->attr("type") + " is not supported (nonReflecting, symmetry, wall)");
    side++;
  }
  *out = in;
  return ECG_OK;
}

extern "C" void ecg_input_free(ecg_input* in) { delete in; }

extern "C" ecg_status ecg_input_case(const ecg_input* in, ecg_case* out) {
  if (!in || !out) return fail(ECG_ERR_INVALID, "ecg_input_case: null argument");
  *out = in->c;
  return ECG_OK;
}

extern "C" const char* ecg_input_run_name(const ecg_input* in) { return in ? in->run_name.c_str() : ""; }

extern "C" ecg_status ecg_input_print_control(const ecg_input* in, int32_t* iter_freq, double* time_freq) {
  if (!in) return fail(ECG_ERR_INVALID, "null input");
  if (iter_freq) *iter_freq = in->iter_freq;
  if (time_freq) *time_freq = in->time_freq;
  return ECG_OK;
}

extern "C" ecg_status ecg_input_output_control(const ecg_input* in, int32_t* binary, int32_t* precision,
                                               int32_t* restart_file) {
  if (!in) return fail(ECG_ERR_INVALID, "null input");
  if (binary) *binary = in->binary;
  if (precision) *precision = in->precision;
  if (restart_file) *restart_file = in->restart_file;
  return ECG_OK;
}

extern "C" ecg_status ecg_restart_fill(const ecg_case* cp, double* const* fields, int64_t ncells) {
  if (!cp || !fields) return fail(ECG_ERR_INVALID, "ecg_restart_fill: null argument");
  const ecg_case& c = *cp;
  int64_t n = (int64_t)c.ncells[0] * c.ncells[1] * c.ncells[2];
  if (ncells != n) return fail(ECG_ERR_INVALID, "ecg_restart_fill: ncells does not match the mesh");
  const int nf = ecg::abi_nfields(c);
  for (int f = 0; f < nf; f++)
    if (!fields[f]) return fail(ECG_ERR_INVALID, "ecg_restart_fill: null field pointer");
  const double eps = c.alpha_null ? 1.e-15 : 0.;
  const int np = c.nphases;
  for (int64_t i = 0; i < n; i++) {
    if (c.model == ECG_MODEL_PTUEQ) {  // ModPTUEq::fulfillState: rho_k from (p, T), then the total energy
      for (int k = 0; k < 2; k++) fields[2 + k][i] = eos_density_pT(c.eos[k], 0., fields[4][i], fields[9][i]);
      fields[8][i] = ptueq_total_energy(c, fields, i);
      continue;
    }
    if (c.model == ECG_MODEL_EULER) {
      const double u0 = fields[2][i], u1 = fields[3][i], u2 = fields[4][i];
      fields[5][i] = ecg::host_eos_e(c.eos[0], eps, fields[0][i], fields[1][i]) + 0.5 * (u0 * u0 + u1 * u1 + u2 * u2);
      continue;
    }
    const double p = fields[2 * np][i];
    double rho = 0., e = 0., ek[ECG_MAX_PHASES];
    for (int k = 0; k < np; k++) {
      double& a = fields[k][i];
      double& r = fields[np + k][i];
      if (eps > 1.e-20) {  // PhaseUEq::verifyAndCorrectPhase src/Models/UEq/PhaseUEq.cpp:355
        if (a < 0.) a = 0.;
        if (a > 1.) a = 1.;
        if (r <= 1.e-15) r = 1.e-15;
      } else {
        if (a < 1e-15) a = 1e-14;
        if (a > 1. - 1e-15) a = 1. - 1e-14;
        if (r < 1.e-15) r = 1.e-14;
      }
      ek[k] = ecg::host_eos_e(c.eos[k], eps, r, ecg::host_eos_fix_p(c.eos[k], p));
    }
    for (int k = 0; k < np; k++) rho += fields[k][i] * fields[np + k][i];
    for (int k = 0; k < np; k++) e += fields[k][i] * fields[np + k][i] / std::max(rho, eps) * ek[k];
    const double u0 = fields[2 * np + 1][i], u1 = fields[2 * np + 2][i], u2 = fields[2 * np + 3][i];
    fields[2 * np + 4][i] = e + 0.5 * (u0 * u0 + u1 * u1 + u2 * u2);
  }
  return ECG_OK;
}

extern "C" const char* ecg_input_eos_name(const ecg_input* in, int32_t k) {
  if (!in || k < 0 || k >= (int)in->eos_names.size()) return "";
  return in->eos_names[k].c_str();
}

namespace {

bool belongs(const Domain& D, const double pos[3]) {
  switch (D.kind) {
    case 0:
      return true;
    case 1:  // GDHalfSpace::belong :77
      if (D.direction >= 0) return pos[D.axis] >= D.origin;
      return pos[D.axis] <= D.origin;
    case 2: {  // GDDisc::belong :78
      double sum = 0.;
      sum += std::pow(pos[D.axis1] - D.c[D.axis1], 2.);
      sum += std::pow(pos[D.axis2] - D.c[D.axis2], 2.);
      return sum <= D.radius * D.radius;
    }
    case 3: {  // GDSphere::belong :64
      double sum = std::pow(pos[0] - D.c[0], 2.) + std::pow(pos[1] - D.c[1], 2.) + std::pow(pos[2] - D.c[2], 2.);
      return sum <= D.radius * D.radius;
    }
    case 4: {  // GDRectangle::belong :81
      const int ax[2] = {D.axis1, D.axis2};
      const double l[2] = {D.l1, D.l2};
      for (int i = 0; i < 2; i++) {
        if (pos[ax[i]] - D.c[ax[i]] < 0) return false;
        if (pos[ax[i]] - D.c[ax[i]] > l[i]) return false;
      }
      return true;
    }
    case 5: {  // GDCuboid::belong :70
      if ((pos[0] - D.c[0]) < 0) return false;
      if ((pos[0] - D.c[0]) > D.lx) return false;
      if ((pos[1] - D.c[1]) < 0) return false;
      if ((pos[1] - D.c[1]) > D.ly) return false;
      if ((pos[2] - D.c[2]) < 0) return false;
      if ((pos[2] - D.c[2]) > D.lz) return false;
      return true;
    }
  }
  return false;
}

}  // namespace

extern "C" ecg_status ecg_input_fill(const ecg_input* in, double* const* fields, int64_t ncells) {
  if (!in || !fields) return fail(ECG_ERR_INVALID, "ecg_input_fill: null argument");
  const ecg_case& c = in->c;
  int64_t n = (int64_t)c.ncells[0] * c.ncells[1] * c.ncells[2];
  if (ncells != n) return fail(ECG_ERR_INVALID, "ecg_input_fill: ncells does not match the mesh");
  const int np = c.nphases;
  const int nf = ecg::abi_nfields(c);
  for (int f = 0; f < nf; f++)
    if (!fields[f]) return fail(ECG_ERR_INVALID, "ecg_input_fill: null field pointer");
  std::vector<double> sz[3], ctr[3];  // cell sizes and centres per axis (stretched or uniform)
  for (int a = 0; a < 3; a++) ecg::axis_cells(c, a, sz[a], ctr[a]);
  const double eps = c.alpha_null ? 1.e-15 : 0.;
  const int nx = c.ncells[0], ny = c.ncells[1];
  for (int64_t i = 0; i < n; i++) {
    int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / ((int64_t)nx * ny));
    const double pos[3] = {ctr[0][ix], ctr[1][iy], ctr[2][iz]};
    const StateIC* S = nullptr;
    for (const Domain& D : in->domains)
      if (belongs(D, pos)) S = &in->states[D.state];
    if (!S) S = &in->states[in->domains[0].state];
    // Cell::completeFulfillState: fulfillState then E = e + |u|^2 / 2 (MixUEq::computeTotalEnergy)
    double E;
    if (c.model == ECG_MODEL_PTUEQ) {
      for (int k = 0; k < 2; k++) {
        fields[k][i] = S->alpha[k];
        fields[2 + k][i] = S->rho[k];
      }
      fields[4][i] = S->p;
      for (int dd = 0; dd < 3; dd++) fields[5 + dd][i] = S->u[dd];
      fields[9][i] = S->T;
      fields[8][i] = ptueq_total_energy(c, fields, i);
    } else if (c.model == ECG_MODEL_KAPILA) {
      double rho = 0., e = 0.;
      double ek[ECG_MAX_PHASES];
      for (int k = 0; k < np; k++) {
        ek[k] = ecg::host_eos_e(c.eos[k], eps, S->rho[k], S->p);
        rho += S->alpha[k] * S->rho[k];
      }
      for (int k = 0; k < np; k++) {
        double Y = S->alpha[k] * S->rho[k] / std::max(rho, eps);
        e += Y * ek[k];
      }
      E = e + 0.5 * (S->u[0] * S->u[0] + S->u[1] * S->u[1] + S->u[2] * S->u[2]);
      for (int k = 0; k < np; k++) {
        fields[k][i] = S->alpha[k];
        fields[np + k][i] = S->rho[k];
      }
      fields[2 * np][i] = S->p;
      for (int dd = 0; dd < 3; dd++) fields[2 * np + 1 + dd][i] = S->u[dd];
      fields[2 * np + 4][i] = E;
      for (int j = 0; j < c.ntransports; j++) fields[2 * np + 5 + j][i] = S->tr[j];
    } else {
      double e = ecg::host_eos_e(c.eos[0], eps, S->rho[0], S->p);
      E = e + 0.5 * (S->u[0] * S->u[0] + S->u[1] * S->u[1] + S->u[2] * S->u[2]);
      fields[0][i] = S->rho[0];
      fields[1][i] = S->p;
      for (int dd = 0; dd < 3; dd++) fields[2 + dd][i] = S->u[dd];
      fields[5][i] = E;
      for (int j = 0; j < c.ntransports; j++) fields[6 + j][i] = S->tr[j];
    }
  }
  return ECG_OK;
}
