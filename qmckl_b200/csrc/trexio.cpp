// qmckl_trexio_read (org/qmckl_trexio.org:1106-1190) for TREXIO files in the
// text backend.
//
// TREXIO (github.com/TREX-CoE/trexio) is a separate library that the
// reference links when it is configured with it; it is not part of the
// reference's sources and not installed here.  Its text backend stores a
// file as a directory with one plain-text file per group (electron.txt,
// nucleus.txt, basis.txt, ao.txt, mo.txt, ...), written by TREXIO 2.x as
//   rank_<array> <rank>            dims_<array> <axis> <extent>
//   <scalar>_isSet <0|1>           <scalar> <value>
//   len_<string> <length>          then a line <string> and the text
//   <array>                        then the values, one per line, in the
//                                  C (row-major) order of the dims
// This file reads that layout for the groups the orbital path needs and
// feeds the values to the context through its own setters in the order and
// with the conversions of the reference's readers:
//   electron  up/dn numbers                      (org/qmckl_trexio.org:118-160)
//   nucleus   number, charges, coordinates 'N'   (164-283)
//   basis/ao  type, shell/prim/ao numbers, nucleus_index and nucleus_shell_num
//             from basis_nucleus_index, r_power (0 when absent), angular
//             momenta, shell_prim_num and shell_prim_index from
//             basis_shell_index, shell factors, exponents, coefficients,
//             primitive factors, ao_normalization as the AO factors (285-1015)
//   mo        number, coefficients [mo][ao]      (1017-1101)
// A path that is not a text-backend directory (an HDF5 file) is reported as
// QMCKL_INVALID_ARG_2, which is what the reference returns when none of its
// backends opens the file; the HDF5 backend needs libtrexio and HDF5.
#include <sys/stat.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "internal.h"

namespace qb {
namespace {

// One group file of the text backend: scalars, strings and arrays by name.
struct TextGroup {
  std::map<std::string, std::string> scalar;            // "<name>" -> value (from "<name> <value>")
  std::map<std::string, std::vector<int64_t>> dims;     // array -> extents
  std::map<std::string, std::vector<std::string>> data; // array or string -> its lines
  bool ok = false;
};

std::vector<std::string> split_ws(const std::string& s) {
  std::istringstream is(s);
  std::vector<std::string> out;
  std::string t;
  while (is >> t) out.push_back(t);
  return out;
}

TextGroup read_group(const std::string& dir, const char* group) {
  TextGroup g;
  std::ifstream f(dir + "/" + group + ".txt");
  if (!f) return g;
  std::vector<std::string> lines;
  for (std::string line; std::getline(f, line);) lines.push_back(line);
  std::map<std::string, int64_t> lens;
  for (size_t i = 0; i < lines.size();) {
    const std::vector<std::string> tok = split_ws(lines[i]);
    if (tok.empty()) { ++i; continue; }
    const std::string& key = tok[0];
    if (tok.size() >= 3 && key.rfind("dims_", 0) == 0) {
      std::vector<int64_t>& d = g.dims[key.substr(5)];
      const size_t axis = (size_t)std::strtoll(tok[1].c_str(), nullptr, 10);
      if (d.size() <= axis) d.resize(axis + 1, 0);
      d[axis] = std::strtoll(tok[2].c_str(), nullptr, 10);
      ++i;
    } else if (tok.size() >= 2 && key.rfind("len_", 0) == 0) {
      lens[key.substr(4)] = std::strtoll(tok[1].c_str(), nullptr, 10);
      ++i;
    } else if (tok.size() >= 2) {
      g.scalar[key] = tok[1];   // rank_*, *_isSet and scalar values
      ++i;
    } else if (g.dims.count(key)) {   // an array: product of its extents, one value per line
      int64_t n = 1;
      for (int64_t e : g.dims[key]) n *= e;
      std::vector<std::string>& v = g.data[key];
      size_t j = i + 1;
      for (; j < lines.size() && (int64_t)v.size() < n; ++j) {
        const std::vector<std::string> t = split_ws(lines[j]);
        for (const std::string& s : t) v.push_back(s);
      }
      i = j;
    } else if (lens.count(key)) {     // a string: the next line (empty when its length is 0)
      std::vector<std::string>& v = g.data[key];
      if (lens[key] > 0 && i + 1 < lines.size()) {
        v.push_back(lines[i + 1]);
        i += 2;
      } else {
        ++i;
      }
    } else {
      ++i;   // an array or string with no values written
    }
  }
  g.ok = true;
  return g;
}

bool is_text_dir(const std::string& path) {
  struct stat st;
  if (stat(path.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) return false;
  struct stat s2;
  return stat((path + "/nucleus.txt").c_str(), &s2) == 0;
}

// Reads of the reference's trexio_read_* calls, with their failure messages.
struct Reader {
  qmckl_context context;
  std::map<std::string, TextGroup> groups;
  std::string dir;

  const TextGroup& group(const char* name) {
    auto it = groups.find(name);
    if (it == groups.end()) it = groups.emplace(name, read_group(dir, name)).first;
    return it->second;
  }
  // scalar `name` of `grp` (also requires <name>_isSet 1)
  bool scalar_i64(const char* grp, const char* name, int64_t* v) {
    const TextGroup& g = group(grp);
    auto s = g.scalar.find(std::string(name) + "_isSet");
    auto x = g.scalar.find(name);
    if (!g.ok || s == g.scalar.end() || s->second != "1" || x == g.scalar.end()) return false;
    *v = std::strtoll(x->second.c_str(), nullptr, 10);
    return true;
  }
  bool string(const char* grp, const char* name, std::string* v) {
    const TextGroup& g = group(grp);
    auto it = g.data.find(name);
    if (!g.ok || it == g.data.end() || it->second.empty()) return false;
    *v = it->second[0];
    return true;
  }
  template <typename T>
  bool array(const char* grp, const char* name, int64_t n, std::vector<T>* v) {
    const TextGroup& g = group(grp);
    auto it = g.data.find(name);
    if (!g.ok || it == g.data.end() || (int64_t)it->second.size() < n) return false;
    v->resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) {
      const char* s = it->second[(size_t)i].c_str();
      char* end = nullptr;
      errno = 0;
      if (std::is_floating_point<T>::value)
        (*v)[(size_t)i] = (T)std::strtod(s, &end);
      else
        (*v)[(size_t)i] = (T)std::strtoll(s, &end, 10);
      if (end == s || errno != 0) return false;
    }
    return true;
  }
  qmckl_exit_code fail(const char* what, const char* msg = "missing or unreadable in the TREXIO text file") {
    return qmckl_failwith(context, QMCKL_FAILURE, what, msg);
  }
};

#define QB_TRY(expr)                         \
  do {                                       \
    const qmckl_exit_code rc_ = (expr);      \
    if (rc_ != QMCKL_SUCCESS) return rc_;    \
  } while (0)

qmckl_exit_code read_electron(Reader& r) {
  int64_t up = 0, dn = 0;
  if (!r.scalar_i64("electron", "electron_up_num", &up)) return r.fail("trexio_read_electron_up_num");
  if (!r.scalar_i64("electron", "electron_dn_num", &dn)) return r.fail("trexio_read_electron_dn_num");
  if (up < 0 || dn < 0) return r.fail("trexio_read_electron_up_num", "negative electron count");
  return qmckl_set_electron_num(r.context, up, dn);
}

qmckl_exit_code read_nucleus(Reader& r) {
  int64_t n = 0;
  if (!r.scalar_i64("nucleus", "nucleus_num", &n) || n <= 0) return r.fail("trexio_read_nucleus_num");
  QB_TRY(qmckl_set_nucleus_num(r.context, n));
  std::vector<double> charge, coord;
  if (!r.array("nucleus", "nucleus_charge", n, &charge)) return r.fail("trexio_read_nucleus_charge");
  QB_TRY(qmckl_set_nucleus_charge(r.context, charge.data(), n));
  if (!r.array("nucleus", "nucleus_coord", 3 * n, &coord)) return r.fail("trexio_read_nucleus_coord");
  return qmckl_set_nucleus_coord(r.context, 'N', coord.data(), 3 * n);
}

qmckl_exit_code read_ao(Reader& r) {
  const qmckl_context c = r.context;
  int64_t nucl_num = 0;
  QB_TRY(qmckl_get_nucleus_num(c, &nucl_num));
  std::string type;
  if (!r.string("basis", "basis_type", &type)) return r.fail("trexio_read_basis_type");
  if (type.empty() || (type[0] != 'G' && type[0] != 'S' && type[0] != 'N'))
    return r.fail("trexio_read_basis_type", "Invalid basis type");
  QB_TRY(qmckl_set_ao_basis_type(c, type[0]));
  int64_t shell_num = 0, prim_num = 0, ao_num = 0;
  if (!r.scalar_i64("basis", "basis_shell_num", &shell_num) || shell_num <= 0)
    return r.fail("trexio_read_basis_shell_num");
  QB_TRY(qmckl_set_ao_basis_shell_num(c, shell_num));
  if (!r.scalar_i64("basis", "basis_prim_num", &prim_num) || prim_num <= 0) return r.fail("trexio_read_basis_prim_num");
  QB_TRY(qmckl_set_ao_basis_prim_num(c, prim_num));
  if (!r.scalar_i64("ao", "ao_num", &ao_num) || ao_num <= 0) return r.fail("trexio_read_ao_num");
  QB_TRY(qmckl_set_ao_basis_ao_num(c, ao_num));
  // basis_nucleus_index: the nucleus of each shell -> first shell of each
  // nucleus (the last loop writes the smallest shell index) and shell counts
  std::vector<int64_t> shell_nucl;
  if (!r.array("basis", "basis_nucleus_index", shell_num, &shell_nucl)) return r.fail("trexio_read_basis_nucleus_index");
  std::vector<int64_t> nucleus_index((size_t)nucl_num, 0), nucleus_shell_num((size_t)nucl_num, 0);
  for (int64_t i = shell_num - 1; i >= 0; --i) {
    const int64_t k = shell_nucl[(size_t)i];
    if (k < 0 || k >= nucl_num) return r.fail("trexio_read_basis_nucleus_index", "Irrelevant data in TREXIO file");
    nucleus_index[(size_t)k] = i;
  }
  QB_TRY(qmckl_set_ao_basis_nucleus_index(c, nucleus_index.data(), shell_num));
  for (int64_t i = 0; i < shell_num; ++i) nucleus_shell_num[(size_t)shell_nucl[(size_t)i]] += 1;
  QB_TRY(qmckl_set_ao_basis_nucleus_shell_num(c, nucleus_shell_num.data(), shell_num));
  std::vector<int32_t> r_power;
  if (!r.array("basis", "basis_r_power", shell_num, &r_power)) r_power.assign((size_t)shell_num, 0);
  QB_TRY(qmckl_set_ao_basis_r_power(c, r_power.data(), shell_num));
  std::vector<int32_t> ang_mom;
  if (!r.array("basis", "basis_shell_ang_mom", shell_num, &ang_mom)) return r.fail("trexio_read_basis_shell_ang_mom");
  QB_TRY(qmckl_set_ao_basis_shell_ang_mom(c, ang_mom.data(), shell_num));
  // basis_shell_index: the shell of each primitive -> primitives per shell
  // and first primitive of each shell
  std::vector<int64_t> prim_shell;
  if (!r.array("basis", "basis_shell_index", prim_num, &prim_shell)) return r.fail("trexio_read_basis_shell_index");
  std::vector<int64_t> shell_prim_num((size_t)shell_num, 0), shell_prim_index((size_t)shell_num, 0);
  for (int64_t i = 0; i < prim_num; ++i) {
    const int64_t k = prim_shell[(size_t)i];
    if (k < 0 || k >= shell_num) {
      char msg[128];
      std::snprintf(msg, sizeof msg, "Irrelevant data in TREXIO file: k = %lld", (long long)k);
      return r.fail("qmckl_trexio_read_basis_shell_index", msg);
    }
    shell_prim_num[(size_t)k] += 1;
  }
  QB_TRY(qmckl_set_ao_basis_shell_prim_num(c, shell_prim_num.data(), shell_num));
  for (int64_t i = prim_num - 1; i >= 0; --i) shell_prim_index[(size_t)prim_shell[(size_t)i]] = i;
  QB_TRY(qmckl_set_ao_basis_shell_prim_index(c, shell_prim_index.data(), shell_num));
  std::vector<double> v;
  if (!r.array("basis", "basis_shell_factor", shell_num, &v)) return r.fail("trexio_read_basis_shell_factor");
  QB_TRY(qmckl_set_ao_basis_shell_factor(c, v.data(), shell_num));
  if (!r.array("basis", "basis_exponent", prim_num, &v)) return r.fail("trexio_read_basis_exponent");
  QB_TRY(qmckl_set_ao_basis_exponent(c, v.data(), prim_num));
  if (!r.array("basis", "basis_coefficient", prim_num, &v)) return r.fail("trexio_read_basis_coefficient");
  QB_TRY(qmckl_set_ao_basis_coefficient(c, v.data(), prim_num));
  if (!r.array("basis", "basis_prim_factor", prim_num, &v)) return r.fail("trexio_read_basis_prim_factor");
  QB_TRY(qmckl_set_ao_basis_prim_factor(c, v.data(), prim_num));
  if (!r.array("ao", "ao_normalization", ao_num, &v)) return r.fail("trexio_read_ao_normalization");
  return qmckl_set_ao_basis_ao_factor(c, v.data(), ao_num);
}

qmckl_exit_code read_mo(Reader& r) {
  int64_t ao_num = 0, mo_num = 0;
  QB_TRY(qmckl_get_ao_basis_ao_num(r.context, &ao_num));
  if (!r.scalar_i64("mo", "mo_num", &mo_num) || mo_num <= 0) return r.fail("trexio_read_mo_num");
  QB_TRY(qmckl_set_mo_basis_mo_num(r.context, mo_num));
  std::vector<double> coef;
  if (!r.array("mo", "mo_coefficient", ao_num * mo_num, &coef)) return r.fail("trexio_read_mo_coefficient");
  return qmckl_set_mo_basis_coefficient(r.context, coef.data(), ao_num * mo_num);
}

}  // namespace
}  // namespace qb

using namespace qb;

extern "C" qmckl_exit_code qmckl_trexio_read(const qmckl_context context, const char* file_name,
                                             const int64_t size_max) {
  if (qmckl_context_check(context) == QMCKL_NULL_CONTEXT) return QMCKL_INVALID_CONTEXT;
  if (file_name == nullptr) return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_trexio_read", "NULL file name");
  if (size_max <= 0) return qmckl_failwith(context, QMCKL_INVALID_ARG_3, "qmckl_trexio_read", "size_max <= 0");
  size_t n = 0;
  while ((int64_t)n < size_max && file_name[n] != '\0') ++n;
  Reader r;
  r.context = context;
  r.dir.assign(file_name, n);
  if (!is_text_dir(r.dir))
    return qmckl_failwith(context, QMCKL_INVALID_ARG_2, "qmckl_trexio_read",
                          "Unable to open TREXIO file: not a TREXIO text-backend directory (this build reads the "
                          "text backend only; the HDF5 backend needs libtrexio)");
  QB_TRY(read_electron(r));
  QB_TRY(read_nucleus(r));
  QB_TRY(read_ao(r));
  return read_mo(r);
}
