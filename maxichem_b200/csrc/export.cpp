// mx_create_from_export: a solver from a folder that maxichem_b200/export.py wrote (meta.txt and tables/*.bin), for a
// caller without Python. The folder is read and checked completely before any CUDA work.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/maxichem_b200.h"

namespace {

struct Table {
  std::string dtype;
  size_t count = 0;
  std::vector<unsigned char> bytes;
};

size_t dtype_size(const std::string& d) {
  if (d == "float64" || d == "int64") return 8;
  if (d == "int32" || d == "uint32") return 4;
  if (d == "uint16" || d == "int16") return 2;
  if (d == "uint8" || d == "int8") return 1;
  return 0;
}

void say(char* err, size_t len, const std::string& msg) {
  if (err && len) std::snprintf(err, len, "mx_create_from_export: %s", msg.c_str());
}

}  // namespace

extern "C" int mx_create_from_export(const char* folder, int device, mx_solver** out, char* err, size_t errlen) {
  if (!folder || !out) {
    say(err, errlen, "null folder or output");
    return MX_ERR_ARGUMENT;
  }
  *out = nullptr;
  const std::string root(folder);
  std::ifstream meta(root + "/meta.txt");
  if (!meta) {
    say(err, errlen, root + "/meta.txt cannot be read");
    return MX_ERR_ARGUMENT;
  }
  std::map<std::string, std::string> kv;
  std::map<std::string, Table> tabs;
  struct Group {
    int threads = 0, sv_rounds = 0, sv_nrows = 0, jac_rounds = 0, jac_nents = 0;
  } groups[2];
  std::string line;
  while (std::getline(meta, line)) {
    std::istringstream in(line);
    std::string key;
    if (!(in >> key)) continue;
    if (key == "table") {
      std::string name;
      Table t;
      if (!(in >> name >> t.dtype >> t.count) || !dtype_size(t.dtype)) {
        say(err, errlen, "a malformed table line: " + line);
        return MX_ERR_NETWORK;
      }
      tabs[name] = t;
    } else if (key == "group") {
      int g = -1;
      Group q;
      if (!(in >> g >> q.threads >> q.sv_rounds >> q.sv_nrows >> q.jac_rounds >> q.jac_nents) || g < 0 || g > 1) {
        say(err, errlen, "a malformed group line: " + line);
        return MX_ERR_NETWORK;
      }
      groups[g] = q;
    } else {
      std::string rest;
      std::getline(in >> std::ws, rest);
      kv[key] = rest;
    }
  }
  auto integer = [&](const char* k, int* v) {
    auto it = kv.find(k);
    if (it == kv.end()) return false;
    char* end = nullptr;
    const long x = std::strtol(it->second.c_str(), &end, 10);
    if (end == it->second.c_str()) return false;
    *v = (int)x;
    return true;
  };
  int format = 0, ns = 0, nr = 0, nrt = 0, nj = 0, nel = 0, nent = 0, troe = 0, eff = 0, piece = 0, npieces = 0;
  if (!integer("export_format", &format) || format != 1) {
    say(err, errlen, "export_format 1 expected");
    return MX_ERR_NETWORK;
  }
  if (!integer("ns", &ns) || !integer("nr", &nr) || !integer("nrt", &nrt) || !integer("nj", &nj) ||
      !integer("nel", &nel) || !integer("n_entries", &nent) || !integer("has_troe", &troe) ||
      !integer("has_eff", &eff) || !integer("sv_piece", &piece) || !integer("n_pieces", &npieces) ||
      kv.find("drift") == kv.end()) {
    say(err, errlen, "meta.txt lacks a size or the drift");
    return MX_ERR_NETWORK;
  }
  const double drift = std::strtod(kv["drift"].c_str(), nullptr);
  // every table with its expected type and length
  struct Want {
    const char* name;
    const char* dtype;
    long count;
  };
  std::vector<Want> want = {
      {"perm", "int32", ns},           {"rx", "uint8", 6L * nr},      {"rc", "float64", 14L * nr},
      {"rf", "int32", nr},             {"nasa", "float64", 18L * ns}, {"atoms", "float64", (long)ns * nel},
      {"sv_ptr", "int32", ns + 1L},    {"sv_term", "uint32", -1},     {"jac_ptr", "int32", nent + 1L},
      {"jac_entry", "uint32", nent},   {"jac_term", "uint32", -1},    {"fill", "uint8", (long)ns * ns},
      {"sv_row_ptr", "int32", ns + 1L}};
  for (int g = 0; g < 2; g++) {
    const Group& q = groups[g];
    static const char* sv[2] = {"sv_stream0", "sv_stream1"};
    static const char* rows[2] = {"sv_rows0", "sv_rows1"};
    static const char* js[2] = {"jac_stream0", "jac_stream1"};
    static const char* jd[2] = {"jac_dst0", "jac_dst1"};
    want.push_back({sv[g], "uint16", (long)q.sv_rounds * q.threads});
    want.push_back({rows[g], "uint16", (long)q.sv_nrows * q.threads});
    want.push_back({js[g], "uint32", (long)q.jac_rounds * q.threads});
    want.push_back({jd[g], "uint16", (long)q.jac_nents * q.threads});
  }
  for (const Want& w : want) {
    auto it = tabs.find(w.name);
    if (it == tabs.end() || it->second.dtype != w.dtype || (w.count >= 0 && (long)it->second.count != w.count)) {
      say(err, errlen, std::string("table ") + w.name + ": " + w.dtype + " of " + std::to_string(w.count) +
                           " entries expected in meta.txt");
      return MX_ERR_NETWORK;
    }
    Table& t = it->second;
    const size_t bytes = t.count * dtype_size(t.dtype);
    std::ifstream f(root + "/tables/" + w.name + ".bin", std::ios::binary);
    t.bytes.resize(bytes ? bytes : 1);
    if (!f || !f.read(reinterpret_cast<char*>(t.bytes.data()), (std::streamsize)bytes) ||
        f.peek() != std::ifstream::traits_type::eof()) {
      say(err, errlen, root + "/tables/" + w.name + ".bin: " + std::to_string(bytes) + " bytes expected");
      return MX_ERR_NETWORK;
    }
  }
  auto ptr = [&](const char* name) { return (const void*)tabs[name].bytes.data(); };
  mx_network n;
  std::memset(&n, 0, sizeof n);
  n.ns = ns;
  n.nr = nr;
  n.nrt = nrt;
  n.nj = nj;
  n.nel = nel;
  n.n_entries = nent;
  n.has_troe = troe;
  n.has_eff = eff;
  n.perm = (const int32_t*)ptr("perm");
  n.rx = (const uint8_t*)ptr("rx");
  n.rc = (const double*)ptr("rc");
  n.rf = (const int32_t*)ptr("rf");
  n.nasa = (const double*)ptr("nasa");
  n.atoms = (const double*)ptr("atoms");
  n.sv_ptr = (const int32_t*)ptr("sv_ptr");
  n.sv_term = (const uint32_t*)ptr("sv_term");
  n.jac_ptr = (const int32_t*)ptr("jac_ptr");
  n.jac_entry = (const uint32_t*)ptr("jac_entry");
  n.jac_term = (const uint32_t*)ptr("jac_term");
  n.fill = (const uint8_t*)ptr("fill");
  n.sv_piece = piece;
  n.n_pieces = npieces;
  n.sv_row_ptr = (const int32_t*)ptr("sv_row_ptr");
  const char* sv[2] = {"sv_stream0", "sv_stream1"};
  const char* rows[2] = {"sv_rows0", "sv_rows1"};
  const char* js[2] = {"jac_stream0", "jac_stream1"};
  const char* jd[2] = {"jac_dst0", "jac_dst1"};
  for (int g = 0; g < 2; g++) {
    n.stream_threads[g] = groups[g].threads;
    n.sv_rounds[g] = groups[g].sv_rounds;
    n.sv_nrows[g] = groups[g].sv_nrows;
    n.jac_rounds[g] = groups[g].jac_rounds;
    n.jac_nents[g] = groups[g].jac_nents;
    n.sv_stream[g] = (const uint16_t*)ptr(sv[g]);
    n.sv_rows[g] = (const uint16_t*)ptr(rows[g]);
    n.jac_stream[g] = (const uint32_t*)ptr(js[g]);
    n.jac_dst[g] = (const uint16_t*)ptr(jd[g]);
  }
  return mx_create(&n, drift, device, out, err, errlen);
}
