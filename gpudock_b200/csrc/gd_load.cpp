// gd_load.cpp -- the reference's input files read into a gd_complex.
//
// Reproduces what linear_dock does before Run: loadProtein / loadLigand /
// loadLHM (gpudocksm-rem-1.2/src/load.C) and the table derivation of
// OptimizeLigand / OptimizeProtein / CopyProteinResidue / OptimizePsp /
// OptimizeKde / OptimizeMcs (util.C:200-458), with the type codes of data.C.
// The arithmetic that shapes the results is kept as the reference does it:
// coordinates parsed as doubles and stored as floats, per-point coordinate
// sums in float in file order, means as float divisions, the ligand centre
// as a float sum over atoms divided by (float)lna.  Capacity limits of the
// reference's fixed arrays are not imposed, except the 70 ligand
// conformations (MAXEN2) that decide which conformations are kept.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <initializer_list>
#include <map>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "gd_common.h"

using gd::fail;

struct gd_loaded {
  std::string ligand_id;
  // ligand
  int lna = 0, n_lig = 0;
  std::vector<float> lx, ly, lz, lc;
  std::vector<int> lt, ln;
  float center[3] = {0.f, 0.f, 0.f};
  // protein
  int pnp = 0, n_prt = 0;
  std::vector<float> px, py, pz, ele, hpp;
  std::vector<int> pt, pc, seq3r, hpcflag;
  // pocket template
  int n_col = 0;
  std::vector<float> psp;
  std::vector<float> kx, ky, kz;
  std::vector<int> kt;
  int pos = 0;
  std::vector<float> mx, my, mz, tcc;
  const gd_enepara *ff = nullptr;
};

namespace {

constexpr int kBadType = 50;       // getLigCode of an unknown name (BADKDE)
constexpr int kMaxLigConf = 70;    // MAXEN2
constexpr int kMcsFields = 256;    // MAXMCS
constexpr float kMcsInvalid = 728492.0f;

// getLigCode (data.C:532-583): Sybyl atom types, index = code.
const char *const kLigNames[GD_NLT] = {"Br",    "C.1", "C.2", "C.3",  "C.ar",  "C.cat",
                                       "Cl",    "F",   "I",   "N.1",  "N.2",   "N.3",
                                       "N.4",   "N.am", "N.ar", "N.pl3", "O.2", "O.3",
                                       "O.co2", "P.3", "S.2", "S.3",  "S.O",   "S.O2"};
// getResCode (data.C:238-287): residue names, index = code.
const char *const kResNames[GD_NRES] = {"ALA", "ARG", "CYS", "PRO", "LEU", "ILE", "GLU",
                                        "HIS", "TRP", "THR", "MET", "ASP", "GLY", "PHE",
                                        "LYS", "GLN", "SER", "ASN", "TYR", "VAL"};
// Side-chain effective points of each residue code as loadProtein pushes
// them (load.C:648-715): count, then {type} and {class}; GLY has none.
struct SidePoints {
  int n;
  int t[2], c[2];
};
const SidePoints kSide[GD_NRES] = {
    {1, {2, 0}, {2, 0}},   {2, {21, 22}, {2, 3}}, {1, {3, 0}, {2, 0}},   {1, {18, 0}, {2, 0}},
    {1, {14, 0}, {2, 0}},  {1, {11, 0}, {2, 0}},  {2, {5, 6}, {2, 3}},   {2, {9, 10}, {2, 3}},
    {2, {26, 27}, {2, 3}}, {1, {24, 0}, {2, 0}},  {2, {15, 16}, {2, 3}}, {1, {4, 0}, {2, 0}},
    {0, {0, 0}, {0, 0}},   {2, {7, 8}, {2, 3}},   {2, {12, 13}, {2, 3}}, {2, {19, 20}, {2, 3}},
    {1, {23, 0}, {2, 0}},  {1, {17, 0}, {2, 0}},  {2, {28, 29}, {2, 3}}, {1, {25, 0}, {2, 0}},
};

// getPntCode (data.C:391-460): protein effective-point names, index = code.
const char *const kPntNames[GD_NPT] = {"CA", "PP", "A1", "C1", "D1", "E1", "E2", "F1",
                                       "F2", "H1", "H2", "I1", "K1", "K2", "L1", "M1",
                                       "M2", "N1", "P1", "Q1", "Q2", "R1", "R2", "S1",
                                       "T1", "V1", "W1", "W2", "Y1", "Y2"};
// getResCodeOne (data.C:290-336): one-letter residue codes, index = code.
const char kResOne[GD_NRES + 1] = "ARCPLIEHWTMDGFKQSNYV";

int lig_code(const std::string &s) {
  for (int i = 0; i < GD_NLT; ++i)
    if (s == kLigNames[i]) return i;
  return kBadType;
}

int pnt_code(const std::string &s) {
  for (int i = 0; i < GD_NPT; ++i)
    if (s == kPntNames[i]) return i;
  return -1;
}

int res_one_code(const std::string &s) {
  if (s.size() != 1) return -1;
  const char *p = std::strchr(kResOne, s[0]);
  return (p && *p) ? (int)(p - kResOne) : -1;
}

int res_code(const std::string &s) {
  for (int i = 0; i < GD_NRES; ++i)
    if (s == kResNames[i]) return i;
  return -1;
}

// substr that tolerates short lines (the reference's fixed columns)
std::string col(const std::string &s, size_t pos, size_t n) {
  return pos < s.size() ? s.substr(pos, n) : std::string();
}

// atof of a field, stored as float (the reference assigns atof to floats)
float fnum(const std::string &s) { return (float)std::atof(s.c_str()); }

bool read_lines(const char *path, std::vector<std::string> *out) {
  std::ifstream f(path);
  if (!f.is_open()) return false;
  std::string line;
  while (std::getline(f, line)) out->push_back(line);
  return true;
}

std::vector<std::string> tokens(const std::string &s) {
  std::vector<std::string> out;
  std::istringstream in(s);
  std::string w;
  while (in >> w) out.push_back(w);
  return out;
}

// Smallest sum of squared deviations of two centred point sets over all
// rotations (weights 1): E = sum |a|^2 + |b|^2 - 2 lambda_max(N), N the 4x4
// symmetric matrix of Horn's quaternion method (J. Opt. Soc. Am. A 4:629,
// 1987) built from the cross-covariance; lambda_max by Jacobi rotations.
// The reference gets the same quantity from Kabsch's u3b (rmsd.f).
double superposed_residual(const std::vector<double> &a, const std::vector<double> &b, int n) {
  double S[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, e0 = 0.0;
  for (int i = 0; i < n; ++i) {
    for (int r = 0; r < 3; ++r) {
      e0 += a[3 * i + r] * a[3 * i + r] + b[3 * i + r] * b[3 * i + r];
      for (int c = 0; c < 3; ++c) S[r][c] += a[3 * i + r] * b[3 * i + c];
    }
  }
  const double sxx = S[0][0], sxy = S[0][1], sxz = S[0][2], syx = S[1][0], syy = S[1][1];
  const double syz = S[1][2], szx = S[2][0], szy = S[2][1], szz = S[2][2];
  double N[4][4] = {{sxx + syy + szz, syz - szy, szx - sxz, sxy - syx},
                    {syz - szy, sxx - syy - szz, sxy + syx, szx + sxz},
                    {szx - sxz, sxy + syx, -sxx + syy - szz, syz + szy},
                    {sxy - syx, szx + sxz, syz + szy, -sxx - syy + szz}};
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, diag = 0.0;
    for (int p = 0; p < 4; ++p) {
      diag += N[p][p] * N[p][p];
      for (int q = p + 1; q < 4; ++q) off += N[p][q] * N[p][q];
    }
    if (off <= 1e-30 * (diag + 1e-300)) break;
    for (int p = 0; p < 4; ++p)
      for (int q = p + 1; q < 4; ++q) {
        if (N[p][q] == 0.0) continue;
        const double theta = (N[q][q] - N[p][p]) / (2.0 * N[p][q]);
        const double t =
            (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 4; ++k) {  // columns p, q
          const double kp = N[k][p], kq = N[k][q];
          N[k][p] = c * kp - s * kq;
          N[k][q] = s * kp + c * kq;
        }
        for (int k = 0; k < 4; ++k) {  // rows p, q
          const double pk = N[p][k], qk = N[q][k];
          N[p][k] = c * pk - s * qk;
          N[q][k] = s * pk + c * qk;
        }
      }
  }
  const double lmax = std::max(std::max(N[0][0], N[1][1]), std::max(N[2][2], N[3][3]));
  return std::max(0.0, e0 - 2.0 * lmax);
}

// ---------------------------------------------------------------------------
// SD file (loadLigand, load.C:100-420)
// ---------------------------------------------------------------------------
gd_status load_ligand(const char *path, const char *molid, gd_loaded *L) {
  std::vector<std::string> lines;
  if (!read_lines(path, &lines)) return fail(GD_EIO, "cannot read %s", path);
  // the reference takes lna / lnb from the counts line of the first record
  // and scans the property lines after its bond block to the end of file
  size_t end = 0;
  while (end < lines.size() && lines[end] != "$$$$") ++end;
  if (end >= lines.size() || end < 10) return fail(GD_EINVAL, "%s: no SD record", path);
  const int lna = std::atoi(col(lines[3], 0, 3).c_str());
  const int lnb = std::atoi(col(lines[3], 3, 3).c_str());
  if (lna < 1 || 4 + (size_t)lna + lnb > lines.size())
    return fail(GD_EINVAL, "%s: bad counts line", path);
  std::vector<int> types;
  std::vector<float> charges;
  std::vector<std::vector<float>> ens;  // raw ensemble coordinates
  const std::string tag = molid ? molid : "MOLID";
  const size_t last = lines.size() - 1;
  for (size_t i = 4 + lna + lnb; i < last; ++i) {
    const std::string &h = lines[i];
    if (!tag.empty() && h.find(tag) != std::string::npos) {
      L->ligand_id = lines[i + 1];
    } else if (h.find("OB_ATOM_TYPES") != std::string::npos) {
      types.clear();
      for (const std::string &w : tokens(lines[i + 1])) types.push_back(lig_code(w));
    } else if (h.find("OB_ATOMIC_CHARGES") != std::string::npos) {
      charges.clear();
      for (const std::string &w : tokens(lines[i + 1])) charges.push_back(fnum(w));
    } else if (h.find("ENSEMBLE_COORDS") != std::string::npos) {
      // one conformation per line, up to an empty line
      while (i + 1 < lines.size() && !lines[i + 1].empty() &&
             (int)ens.size() < kMaxLigConf) {
        ++i;
        std::vector<float> c;
        for (const std::string &w : tokens(lines[i])) c.push_back(fnum(w));
        c.resize(3 * (size_t)lna, 0.f);
        ens.push_back(c);
      }
      ++i;  // the line that ended the block
    }
  }
  if ((int)types.size() < lna)
    return fail(GD_EINVAL, "%s: OB_ATOM_TYPES has %zu of %d atoms", path, types.size(), lna);
  if ((int)charges.size() < lna)
    return fail(GD_EINVAL, "%s: OB_ATOMIC_CHARGES has %zu of %d atoms", path, charges.size(), lna);

  // default pose from the atom block; centre = float mean over atoms
  std::vector<float> native(3 * (size_t)lna);
  float cen[3] = {0.f, 0.f, 0.f};
  for (int a = 0; a < lna; ++a) {
    const std::string &s = lines[4 + a];
    native[3 * a] = fnum(col(s, 0, 10));
    native[3 * a + 1] = fnum(col(s, 10, 10));
    native[3 * a + 2] = fnum(col(s, 20, 10));
    for (int k = 0; k < 3; ++k) cen[k] += native[3 * a + k];
  }
  for (int k = 0; k < 3; ++k) cen[k] /= (float)lna;
  for (int a = 0; a < lna; ++a)
    for (int k = 0; k < 3; ++k) native[3 * a + k] -= cen[k];

  // conformations: the default one, then every ensemble conformation (centred
  // on its own mean) more than 0.1 A RMSD from it after superposition
  std::vector<std::vector<float>> confs(1, native);
  std::vector<double> ref(3 * (size_t)lna), mob(3 * (size_t)lna);
  for (size_t j = 0; j < native.size(); ++j) ref[j] = native[j];
  for (const std::vector<float> &e : ens) {
    float mc[3] = {0.f, 0.f, 0.f};
    for (int a = 0; a < lna; ++a)
      for (int k = 0; k < 3; ++k) mc[k] += e[3 * a + k];
    for (int k = 0; k < 3; ++k) mc[k] /= (float)lna;
    std::vector<float> m(3 * (size_t)lna);
    for (int a = 0; a < lna; ++a)
      for (int k = 0; k < 3; ++k) m[3 * a + k] = e[3 * a + k] - mc[k];
    for (size_t j = 0; j < m.size(); ++j) mob[j] = m[j];
    const float rms = (float)superposed_residual(mob, ref, lna);
    if (std::sqrt(rms / (float)lna) > 0.1) confs.push_back(m);  // as load.C:399-401
    if ((int)confs.size() >= kMaxLigConf) break;
  }

  L->lna = lna;
  L->n_lig = (int)confs.size();
  for (const std::vector<float> &c : confs)
    for (int a = 0; a < lna; ++a) {
      L->lx.push_back(c[3 * a]);
      L->ly.push_back(c[3 * a + 1]);
      L->lz.push_back(c[3 * a + 2]);
    }
  L->lt.assign(types.begin(), types.begin() + lna);
  L->lc.assign(charges.begin(), charges.begin() + lna);
  L->ln.resize(lna);
  for (int a = 0; a < lna; ++a) L->ln[a] = a;
  for (int k = 0; k < 3; ++k) L->center[k] = cen[k];
  return GD_OK;
}

// ---------------------------------------------------------------------------
// PDB ensemble (loadProtein, load.C:595-990; CopyProteinResidue, util.C)
// ---------------------------------------------------------------------------
struct Atom {
  int serial;        // residue serial number (columns 23-26)
  char name[5];      // atom name (columns 13-16)
  float x, y, z;
  int model;         // ENDMDL lines before it
};

bool is_atom(const std::string &s) { return s.size() > 53 && s.compare(0, 6, "ATOM  ") == 0; }
bool is_endmdl(const std::string &s) { return s.compare(0, 6, "ENDMDL") == 0; }

gd_status load_protein(const char *path, const gd_enepara_raw *raw, unsigned flags,
                       gd_loaded *L) {
  std::vector<std::string> lines;
  if (!read_lines(path, &lines)) return fail(GD_EIO, "cannot read %s", path);
  int n_models = 0;
  for (const std::string &s : lines) n_models += is_endmdl(s) ? 1 : 0;
  if (n_models == 0) return fail(GD_EINVAL, "%s: no MODEL / ENDMDL models", path);

  // points of the first model: per CA a CA point, from the third residue on
  // the peptide-plane point of the previous residue, and the side chain
  std::vector<int> seq3, pr, pt, pd, pc;
  auto push = [&](int r, int t, int d, int c) {
    pr.push_back(r);
    pt.push_back(t);
    pd.push_back(d);
    pc.push_back(c);
  };
  for (const std::string &s : lines) {
    if (is_endmdl(s)) break;
    if (!is_atom(s) || s.compare(12, 4, " CA ") != 0) continue;
    const int d = res_code(s.substr(17, 3));
    if (d < 0) return fail(GD_EINVAL, "%s: unknown residue %s", path, s.substr(17, 3).c_str());
    const int pnr = (int)seq3.size();
    seq3.push_back(std::atoi(s.substr(22, 4).c_str()));
    push(pnr, 0, d, 0);
    if (pnr > 1) push(pnr - 1, 1, d, 1);
    for (int k = 0; k < kSide[d].n; ++k) push(pnr, kSide[d].t[k], d, kSide[d].c[k]);
  }
  const int pnr = (int)seq3.size();
  const int pnp = (int)pt.size();
  if (pnp == 0) return fail(GD_EINVAL, "%s: no CA atoms", path);

  // every ATOM record with its model number, by residue serial, file order
  std::vector<Atom> atoms;
  std::map<int, std::vector<int>> by_serial;
  {
    int model = 0;
    for (const std::string &s : lines) {
      if (is_endmdl(s)) {
        ++model;
        continue;
      }
      if (!is_atom(s)) continue;
      Atom a;
      a.serial = std::atoi(s.substr(22, 4).c_str());
      std::memcpy(a.name, s.data() + 12, 4);
      a.name[4] = 0;
      a.x = fnum(s.substr(30, 8));
      a.y = fnum(s.substr(38, 8));
      a.z = fnum(s.substr(46, 8));
      a.model = model;
      by_serial[a.serial].push_back((int)atoms.size());
      atoms.push_back(a);
    }
  }
  auto named = [](const Atom &a, const char *n) { return std::strcmp(a.name, n) == 0; };
  auto backbone = [&](const Atom &a) {
    return named(a, " N  ") || named(a, " CA ") || named(a, " C  ") || named(a, " O  ");
  };
  auto in_list = [](int t, std::initializer_list<int> l) {
    return std::find(l.begin(), l.end(), t) != l.end();
  };

  L->pnp = pnp;
  L->n_prt = n_models;
  // a point none of whose atoms is present in a model is left at 0 there
  // (the reference leaves that coordinate unset)
  L->px.assign((size_t)n_models * pnp, 0.f);
  L->py.assign((size_t)n_models * pnp, 0.f);
  L->pz.assign((size_t)n_models * pnp, 0.f);
  for (int p = 0; p < pnp; ++p) {
    const int r = pr[p], t = pt[p];
    const int s3 = seq3[r];
    const bool pp = t == 1 && r > 0 && r < pnr - 1;
    // the previous residue of a peptide-plane point: its serial in the first
    // two models; later models see serial 0 in the reference, whose loader
    // reads it from a conformation it has not filled yet (zeroed memory),
    // unless GD_LOAD_PEPTIDE_ALL_MODELS asks for the rule in every model
    const int s6 = pp ? seq3[r - 1] : 0;
    const int s6_late = (flags & GD_LOAD_PEPTIDE_ALL_MODELS) ? s6 : 0;
    std::vector<int> idx;
    {
      std::vector<int> serials(1, s3);
      if (pp) {
        serials.push_back(s6);
        serials.push_back(s6_late);
      }
      std::sort(serials.begin(), serials.end());
      serials.erase(std::unique(serials.begin(), serials.end()), serials.end());
      for (int sv : serials) {  // the residues' records, merged in file order
        auto f = by_serial.find(sv);
        if (f == by_serial.end()) continue;
        std::vector<int> m(idx.size() + f->second.size());
        std::merge(idx.begin(), idx.end(), f->second.begin(), f->second.end(), m.begin());
        idx.swap(m);
      }
    }
    std::vector<float> sx(n_models + 1, 0.f), sy(n_models + 1, 0.f), sz(n_models + 1, 0.f);
    std::vector<float> sn(n_models + 1, 0.f);
    for (int i : idx) {
      const Atom &a = atoms[i];
      bool take = false;
      if (a.serial == s3) {
        if (t == 0)
          take = named(a, " CA ");
        else if (in_list(t, {2, 3, 4, 11, 14, 17, 18, 23, 24, 25}))
          take = !backbone(a);
        else if (in_list(t, {5, 7, 9, 12, 15, 19, 21, 26, 28}))
          take = !backbone(a) && !named(a, " CB ") && !named(a, " CG ");
        else if (in_list(t, {6, 8, 10, 13, 16, 20, 22, 27, 29}))
          take = named(a, " CB ") || named(a, " CG ");
      }
      const int prev = a.model < 2 ? s6 : s6_late;
      if (pp && ((a.serial == s3 && named(a, " N  ")) ||
                 (a.serial == prev && (named(a, " C  ") || named(a, " O  ")))))
        take = true;
      if (!take) continue;
      sx[a.model] += a.x;
      sy[a.model] += a.y;
      sz[a.model] += a.z;
      sn[a.model] += 1.0f;
    }
    for (int m = 0; m < n_models; ++m)
      if (sn[m] > 0.0f) {
        L->px[(size_t)m * pnp + p] = sx[m] / sn[m];
        L->py[(size_t)m * pnp + p] = sy[m] / sn[m];
        L->pz[(size_t)m * pnp + p] = sz[m] / sn[m];
      }
  }
  // point properties (CopyProteinResidue, util.C:253-275; no reordering)
  L->pt = pt;
  L->pc = pc;
  L->ele.resize(pnp);
  L->hpp.resize(pnp);
  L->seq3r.resize(pnp);
  L->hpcflag.resize(pnp);
  for (int p = 0; p < pnp; ++p) {
    const int d = pd[p];
    L->ele[p] = raw->ele[pt[p] == 0 ? d + 30 : pt[p]];
    L->hpp[p] = raw->hpp[d];
    L->seq3r[p] = seq3[pr[p]];
    L->hpcflag[p] = ((pc[p] == 0 && d == 12) || pc[p] == 2) ? 1 : 0;
  }
  return GD_OK;
}

// ---------------------------------------------------------------------------
// Pocket template .ff (loadLHM, load.C:1011-1126; OptimizePsp / Kde / Mcs)
// ---------------------------------------------------------------------------
gd_status load_lhm(const char *path, const char *ligand_id, gd_loaded *L) {
  std::vector<std::string> lines;
  if (!read_lines(path, &lines)) return fail(GD_EIO, "cannot read %s", path);
  const std::string want = ligand_id ? ligand_id : "";
  int max_seq = 0;
  for (int s : L->seq3r) max_seq = std::max(max_seq, s);
  // the kernel reads psp[type][seq3r] for protein points only: entries of
  // other residues cannot be reached
  L->n_col = max_seq + 1;
  L->psp.assign((size_t)GD_NLT * L->n_col, 0.f);
  for (const std::string &s : lines) {
    if (s.size() <= 3) continue;
    const std::string key = s.substr(0, 3);
    if (key == "KDE") {
      const std::vector<std::string> w = tokens(s);
      if (w.size() < 5) return fail(GD_EINVAL, "%s: short KDE line", path);
      const int t = lig_code(w[1]);
      if (t >= GD_NLT) continue;  // matches no ligand atom
      L->kt.push_back(t);
      L->kx.push_back(fnum(w[2]));
      L->ky.push_back(fnum(w[3]));
      L->kz.push_back(fnum(w[4]));
    } else if (key == "PSP") {
      const std::vector<std::string> w = tokens(s);
      if (w.size() < 4) return fail(GD_EINVAL, "%s: short PSP line", path);
      const int seq = std::atoi(w[1].c_str()), t = lig_code(w[2]);
      if (t < GD_NLT && seq >= 0 && seq < L->n_col)
        L->psp[(size_t)t * L->n_col + seq] = fnum(w[3]);
    } else if (key == "MCS") {
      // every MCS line is a record; those of other ligands stay empty
      const std::vector<std::string> w = tokens(s);
      const size_t base = L->mx.size();
      L->mx.resize(base + kMcsFields, kMcsInvalid);
      L->my.resize(base + kMcsFields, kMcsInvalid);
      L->mz.resize(base + kMcsFields, kMcsInvalid);
      L->tcc.push_back(0.f);
      L->pos += 1;
      if (w.size() >= 4 && w[1] == want) {
        L->tcc.back() = fnum(w[2]);
        const int total = std::atoi(w[3].c_str());
        for (int k = 0; k < total; ++k) {
          if (w.size() < (size_t)(k * 4 + 8)) return fail(GD_EINVAL, "%s: short MCS line", path);
          const int f = std::atoi(w[k * 4 + 4].c_str());
          if (f < 0 || f >= kMcsFields) return fail(GD_EINVAL, "%s: MCS field %d", path, f);
          L->mx[base + f] = fnum(w[k * 4 + 5]);
          L->my[base + f] = fnum(w[k * 4 + 6]);
          L->mz[base + f] = fnum(w[k * 4 + 7]);
        }
      }
    }
  }
  return GD_OK;
}

// The force-field parameter file (loadEnePara, load.C:1139-1324): tagged
// lines of whitespace-separated fields, values by atof stored as floats, a
// missing field reading as 0.  Unknown point, ligand or residue names are
// errors (the reference exits on the first and the third and indexes past
// its tables with the second).  Afterwards the residue hydrophobicities are
// rescaled to [-1, 1]: difference and quotient in float, "* 2 - 1" in
// double, clamped (load.C:1297-1323).
gd_status load_ff_params(const char *path, gd_enepara_raw *R) {
  std::vector<std::string> lines;
  if (!read_lines(path, &lines)) return fail(GD_EIO, "cannot open %s", path);
  for (size_t li = 0; li < lines.size(); ++li) {
    const std::string &line = lines[li];
    if (line.size() <= 3) continue;
    const std::string tag = line.substr(0, 3);
    const std::vector<std::string> w = tokens(line);
    auto val = [&](size_t k) { return k < w.size() ? fnum(w[k]) : 0.0f; };
    auto name = [&](size_t k) { return k < w.size() ? w[k] : std::string(); };
    auto bad = [&](const char *what) {
      return fail(GD_EINVAL, "%s line %zu: unknown %s", path, li + 1, what);
    };
    if (tag == "VDW" || tag == "PMF" || tag == "HDB") {
      const int p = pnt_code(name(1)), l = lig_code(name(2));
      if (p < 0) return bad("point type");
      if (l >= GD_NLT) return bad("ligand type");
      float(*t)[GD_NLT][2] = tag == "VDW" ? R->vdw : tag == "PMF" ? R->pmf : R->hdb;
      t[p][l][0] = val(3);
      t[p][l][1] = val(4);
    } else if (tag == "PLJ") {
      for (int k = 0; k < 3; ++k) R->lj[k] = val(1 + k);
    } else if (tag == "ELE") {
      // "<res>C": the residue's backbone class (ele[30 + residue]), else a
      // point type
      const std::string n = name(1);
      if (n.size() >= 2 && n[1] == 'C') {
        const int r = res_one_code(n.substr(0, 1));
        if (r < 0) return bad("residue");
        R->ele[GD_NPT + r] = val(2);
      } else {
        const int p = pnt_code(n);
        if (p < 0) return bad("point type");
        R->ele[p] = val(2);
      }
    } else if (tag == "PEL") {
      for (int k = 0; k < 2; ++k) R->el[k] = val(1 + k);
    } else if (tag == "HPP") {
      const int r = res_one_code(name(1));
      if (r < 0) return bad("residue");
      R->hpp[r] = val(2);
    } else if (tag == "HPL") {
      const int l = lig_code(name(1));
      if (l >= GD_NLT) return bad("ligand type");
      R->hpl[l][0] = val(2);
      R->hpl[l][1] = val(3);
    } else if (tag == "WEI") {
      for (int k = 0; k < GD_NTERM; ++k) R->w[k] = val(1 + k);
    } else if (tag == "KDE") {
      R->kde = val(1);
    }
  }
  float lo = 1e6f, hi = -1e6f;
  for (int r = 0; r < GD_NRES; ++r) {
    lo = std::min(lo, R->hpp[r]);
    hi = std::max(hi, R->hpp[r]);
  }
  for (int r = 0; r < GD_NRES; ++r) {
    const float q = (R->hpp[r] - lo) / (hi - lo);
    float h = (float)((double)q * 2.0 - 1.0);
    if (h < -1.0f) h = -1.0f;
    if (h > 1.0f) h = 1.0f;
    R->hpp[r] = h;
  }
  return GD_OK;
}

// One value per line from its first 30 characters, read as a float by a
// stream (which leaves 0 where no number parses and the largest float on
// overflow), for the first GD_NTERM lines: loadWeight and loadNorPara
// (load.C:1326-1419).  Later lines are ignored (the reference writes them
// past its arrays).
gd_status load_column(const char *path, float *dst) {
  std::vector<std::string> lines;
  if (!read_lines(path, &lines)) return fail(GD_EIO, "cannot open %s", path);
  for (size_t i = 0; i < lines.size() && i < (size_t)GD_NTERM; ++i) {
    std::istringstream in(col(lines[i], 0, 30));
    float v = 0.0f;
    in >> v;
    dst[i] = v;
  }
  return GD_OK;
}

}  // namespace

extern "C" gd_status gd_load_enepara(const char *ff, const char *weights, const char *nor_a,
                                     const char *nor_b, gd_enepara_raw *out) {
  if (!ff || !out) return fail(GD_EINVAL, "gd_load_enepara: NULL argument");
  gd_enepara_raw R;
  std::memset(&R, 0, sizeof(R));
  gd_status st;
  try {
    st = load_ff_params(ff, &R);
    if (st == GD_OK && weights) st = load_column(weights, R.w);
    if (st == GD_OK && nor_a) st = load_column(nor_a, R.a_para);
    if (st == GD_OK && nor_b) st = load_column(nor_b, R.b_para);
  } catch (const std::bad_alloc &) {
    st = fail(GD_ENOMEM, "host allocation");
  }
  if (st == GD_OK) *out = R;
  return st;
}

extern "C" gd_status gd_load(const char *pdb, const char *sdf, const char *lhm,
                             const char *ligand_id, const char *molid,
                             const gd_enepara_raw *raw, const gd_enepara *ff, unsigned flags,
                             gd_loaded **out) {
  if (!pdb || !sdf || !lhm || !raw || !out) return fail(GD_EINVAL, "gd_load: NULL argument");
  *out = nullptr;
  gd_loaded *L = new (std::nothrow) gd_loaded;
  if (!L) return fail(GD_ENOMEM, "host allocation");
  gd_status st;
  try {
    st = load_ligand(sdf, molid, L);
    if (st == GD_OK) st = load_protein(pdb, raw, flags, L);
    if (st == GD_OK) st = load_lhm(lhm, ligand_id, L);
  } catch (const std::bad_alloc &) {
    st = fail(GD_ENOMEM, "host allocation");
  } catch (const std::exception &e) {
    st = fail(GD_EINVAL, "malformed input: %s", e.what());
  }
  if (st != GD_OK) {
    delete L;
    return st;
  }
  L->ff = ff;
  *out = L;
  return GD_OK;
}

extern "C" gd_status gd_loaded_complex(const gd_loaded *L, gd_complex *cx) {
  if (!L || !cx) return fail(GD_EINVAL, "gd_loaded_complex: NULL argument");
  std::memset(cx, 0, sizeof(*cx));
  cx->lig.lna = L->lna;
  cx->lig.n_conf = L->n_lig;
  cx->lig.x = L->lx.data();
  cx->lig.y = L->ly.data();
  cx->lig.z = L->lz.data();
  cx->lig.t = L->lt.data();
  cx->lig.c = L->lc.data();
  cx->lig.n = L->ln.data();
  // OptimizeLigand: the ligand centre is the pocket centre, which starts as
  // the default pose's centre; OptimizeProtein gives it to the protein
  for (int k = 0; k < 3; ++k) {
    cx->lig.center[k] = L->center[k];
    cx->prt.pocket_center[k] = L->center[k];
  }
  cx->prt.pnp = L->pnp;
  cx->prt.n_conf = L->n_prt;
  cx->prt.x = L->px.data();
  cx->prt.y = L->py.data();
  cx->prt.z = L->pz.data();
  cx->prt.t = L->pt.data();
  cx->prt.c = L->pc.data();
  cx->prt.ele = L->ele.data();
  cx->prt.seq3r = L->seq3r.data();
  cx->prt.c0_and_d12_or_c2 = L->hpcflag.data();
  cx->prt.hpp = L->hpp.data();
  cx->psp.n_col = L->n_col;
  cx->psp.psp = L->psp.data();
  cx->kde.pnk = (int)L->kt.size();
  cx->kde.x = L->kx.data();
  cx->kde.y = L->ky.data();
  cx->kde.z = L->kz.data();
  cx->kde.t = L->kt.data();
  cx->mcs.pos = L->pos;
  cx->mcs.n_field = kMcsFields;
  cx->mcs.x = L->mx.data();
  cx->mcs.y = L->my.data();
  cx->mcs.z = L->mz.data();
  cx->mcs.tcc = L->tcc.data();
  cx->ff = L->ff;
  return GD_OK;
}

extern "C" const char *gd_loaded_ligand_id(const gd_loaded *L) {
  return L ? L->ligand_id.c_str() : "";
}

extern "C" gd_status gd_loaded_free(gd_loaded *L) {
  delete L;
  return GD_OK;
}
