// mm_ovf.cu -- OOMMF OVF 2.0 files of a magnetisation (host code only).
//
// The format MicroMagnetic.jl writes and reads (src/ovf2.jl:60-300): a text
// header of "# key: value" lines, then one data block in cell order (x
// fastest, then y, then z) with the three components of a cell together:
//   "Data Binary 8": the check value 123456789012345.0 as float64, then 3N
//                    little-endian float64, a newline;
//   "Data Binary 4": the check value 1234567.0 as float32, then 3N float32;
//   "Data Text":     one line "mx my mz" per cell.
// This is the AoS order of mm_set_m / mm_get_m, so a file is a direct image
// of the boundary array.
#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mmcuda.h"

namespace mm {
int set_last_error(int code, const char* msg);  // mm_api.cu
}

namespace {

int err(int code, const std::string& msg) { return mm::set_last_error(code, msg.c_str()); }

// save_ovf / read_ovf append ".ovf" to a name without it (src/ovf2.jl:70-72, 247-249)
std::string with_ext(const char* path) {
  std::string p(path);
  if (p.size() < 4 || p.compare(p.size() - 4, 4, ".ovf") != 0) p += ".ovf";
  return p;
}

// shortest decimal that reads back to the same double
std::string num(double v) {
  char b[64];
  auto r = std::to_chars(b, b + sizeof(b), v);
  return std::string(b, r.ptr);
}

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

bool little_endian() {
  const uint16_t one = 1;
  unsigned char c;
  std::memcpy(&c, &one, 1);
  return c == 1;
}

// one line without its '\n'; false at end of file with nothing read
bool read_line(FILE* f, std::string& out) {
  out.clear();
  int c;
  while ((c = fgetc(f)) != EOF) {
    if (c == '\n') return true;
    out.push_back(static_cast<char>(c));
  }
  return !out.empty();
}

std::string trim(const std::string& s) {
  size_t a = s.find_first_not_of(" \t\r"), b = s.find_last_not_of(" \t\r");
  return a == std::string::npos ? std::string() : s.substr(a, b - a + 1);
}

std::string lower(std::string s) {
  for (char& c : s) c = static_cast<char>(tolower(static_cast<unsigned char>(c)));
  return s;
}

struct Header {
  int64_t nx = 0, ny = 0, nz = 0;
  double dx = 0, dy = 0, dz = 0;
  int valuedim = 3;
  int type = -1;  // mm_ovf_type
  std::string title;
};

// header of read_ovf(fname)  src/ovf2.jl:246-291; leaves f at the first data byte
int read_header(FILE* f, Header& h) {
  std::string line;
  if (!read_line(f, line) || line.rfind("# OOMMF OVF 2", 0) != 0)
    return err(MM_ERR_ARG, "Input is not a OVF2 file.");
  while (read_line(f, line)) {
    if (line.size() < 2 || line[0] != '#') continue;
    const size_t colon = line.find(':');
    if (colon == std::string::npos) continue;
    const std::string key = lower(trim(line.substr(1, colon - 1)));
    const std::string val = trim(line.substr(colon + 1));
    if (key == "title") h.title = val;
    else if (key == "xnodes") h.nx = std::atoll(val.c_str());
    else if (key == "ynodes") h.ny = std::atoll(val.c_str());
    else if (key == "znodes") h.nz = std::atoll(val.c_str());
    else if (key == "xstepsize") h.dx = std::atof(val.c_str());
    else if (key == "ystepsize") h.dy = std::atof(val.c_str());
    else if (key == "zstepsize") h.dz = std::atof(val.c_str());
    else if (key == "valuedim") h.valuedim = std::atoi(val.c_str());
    else if (key == "begin" && lower(val).rfind("data", 0) == 0) {
      const std::string kind = lower(trim(val.substr(4)));
      if (kind == "binary 8") h.type = MM_OVF_BINARY8;
      else if (kind == "binary 4") h.type = MM_OVF_BINARY4;
      else if (kind == "text") h.type = MM_OVF_TEXT;
      else return err(MM_ERR_ARG, "Data format error!");
      break;
    }
  }
  if (h.type < 0) return err(MM_ERR_ARG, "OVF2 file has no data segment");
  if (h.nx < 1 || h.ny < 1 || h.nz < 1) return err(MM_ERR_ARG, "OVF2 header has no valid xnodes/ynodes/znodes");
  if (h.nx > INT32_MAX || h.ny > INT32_MAX || h.nz > INT32_MAX) return err(MM_ERR_ARG, "OVF2 mesh too large");
  // 3 * xnodes * ynodes * znodes must fit int64: checked by division before
  // any product is formed (the header is untrusted input)
  constexpr int64_t kMaxCells = INT64_MAX / 3;
  if (h.nx > kMaxCells / h.ny || h.nx * h.ny > kMaxCells / h.nz) return err(MM_ERR_ARG, "OVF2 mesh too large");
  if (h.valuedim != 3) return err(MM_ERR_UNSUPPORTED, "OVF2 valuedim other than 3");
  return MM_OK;
}

int read_data(FILE* f, const Header& h, double* out) {
  const int64_t n3 = 3 * h.nx * h.ny * h.nz;
  if (h.type == MM_OVF_BINARY8 || h.type == MM_OVF_BINARY4) {
    if (!little_endian()) return err(MM_ERR_UNSUPPORTED, "big-endian host");
    if (h.type == MM_OVF_BINARY8) {
      double chk = 0;
      if (fread(&chk, 8, 1, f) != 1 || chk != 123456789012345.0)
        return err(MM_ERR_ARG, "OVF2 Binary 8 check value missing");
      if (fread(out, 8, static_cast<size_t>(n3), f) != static_cast<size_t>(n3))
        return err(MM_ERR_ARG, "OVF2 data block is shorter than 3*xnodes*ynodes*znodes values");
    } else {
      float chk = 0;
      if (fread(&chk, 4, 1, f) != 1 || chk != 1234567.0f)
        return err(MM_ERR_ARG, "OVF2 Binary 4 check value missing");
      std::vector<float> tmp(static_cast<size_t>(n3));
      if (fread(tmp.data(), 4, tmp.size(), f) != tmp.size())
        return err(MM_ERR_ARG, "OVF2 data block is shorter than 3*xnodes*ynodes*znodes values");
      for (int64_t i = 0; i < n3; ++i) out[i] = tmp[static_cast<size_t>(i)];
    }
    return MM_OK;
  }
  // Data Text: whitespace-separated numbers up to the next '#' line
  int64_t i = 0;
  std::string line;
  while (read_line(f, line)) {
    if (!line.empty() && line[0] == '#') break;
    const char* p = line.c_str();
    while (*p) {
      while (*p == ' ' || *p == '\t' || *p == '\r') ++p;
      if (!*p) break;
      char* end = nullptr;
      const double v = std::strtod(p, &end);
      if (end == p) return err(MM_ERR_ARG, "OVF2 text data: not a number");
      if (i >= n3) return err(MM_ERR_ARG, "OVF2 text data: more values than 3*xnodes*ynodes*znodes");
      out[i++] = v;
      p = end;
    }
  }
  if (i != n3) return err(MM_ERR_ARG, "OVF2 text data: fewer values than 3*xnodes*ynodes*znodes");
  return MM_OK;
}

}  // namespace

extern "C" {

// save_ovf(ovf::OVF2, fname; type)  src/ovf2.jl:70-153
int mm_ovf_write(const char* path, const mm_mesh_desc* mesh, const double* m_aos, int type, const char* title) {
  if (!path || !mesh || !m_aos) return err(MM_ERR_ARG, "mm_ovf_write: null argument");
  if (mesh->nx < 1 || mesh->ny < 1 || mesh->nz < 1) return err(MM_ERR_ARG, "mm_ovf_write: bad mesh");
  if (type != MM_OVF_BINARY8 && type != MM_OVF_BINARY4 && type != MM_OVF_TEXT)
    return err(MM_ERR_ARG, "mm_ovf_write: type must be MM_OVF_BINARY8, MM_OVF_BINARY4 or MM_OVF_TEXT");
  if (type != MM_OVF_TEXT && !little_endian()) return err(MM_ERR_UNSUPPORTED, "big-endian host");
  const std::string fn = with_ext(path);
  File F;
  F.f = fopen(fn.c_str(), "wb");
  if (!F.f) return err(MM_ERR_ARG, "cannot open " + fn + " for writing: " + std::strerror(errno));
  const int64_t nx = mesh->nx, ny = mesh->ny, nz = mesh->nz, n3 = 3 * nx * ny * nz;
  const double dx = mesh->dx, dy = mesh->dy, dz = mesh->dz;
  std::string hd = "# OOMMF OVF 2.0\n";
  auto kv = [&](const char* k, const std::string& v) { hd += std::string("# ") + k + ": " + v + "\n"; };
  kv("Segment count", "1");
  kv("Begin", "Segment");
  kv("Begin", "Header");
  kv("Title", title ? title : "");
  kv("meshtype", "rectangular");
  kv("meshunit", "m");
  kv("xmin", "0");
  kv("ymin", "0");
  kv("zmin", "0");
  kv("xmax", num(nx * dx));
  kv("ymax", num(ny * dy));
  kv("zmax", num(nz * dz));
  kv("valuedim", "3");
  kv("valuelabels", "m_x m_y m_z");
  kv("valueunits", "1 1 1");
  kv("xbase", num(dx / 2));
  kv("ybase", num(dy / 2));
  kv("zbase", num(dz / 2));
  kv("xnodes", std::to_string(nx));
  kv("ynodes", std::to_string(ny));
  kv("znodes", std::to_string(nz));
  kv("xstepsize", num(dx));
  kv("ystepsize", num(dy));
  kv("zstepsize", num(dz));
  kv("End", "Header");
  bool ok = fwrite(hd.data(), 1, hd.size(), F.f) == hd.size();
  if (type == MM_OVF_BINARY8) {
    const double chk = 123456789012345.0;
    ok = ok && fputs("# Begin: Data Binary 8\n", F.f) >= 0;
    ok = ok && fwrite(&chk, 8, 1, F.f) == 1;
    ok = ok && fwrite(m_aos, 8, static_cast<size_t>(n3), F.f) == static_cast<size_t>(n3);
    ok = ok && fputs("\n# End: Data Binary 8\n", F.f) >= 0;
  } else if (type == MM_OVF_BINARY4) {
    const float chk = 1234567.0f;
    std::vector<float> tmp(static_cast<size_t>(n3));
    for (int64_t i = 0; i < n3; ++i) tmp[static_cast<size_t>(i)] = static_cast<float>(m_aos[i]);
    ok = ok && fputs("# Begin: Data Binary 4\n", F.f) >= 0;
    ok = ok && fwrite(&chk, 4, 1, F.f) == 1;
    ok = ok && fwrite(tmp.data(), 4, tmp.size(), F.f) == tmp.size();
    ok = ok && fputs("\n# End: Data Binary 4\n", F.f) >= 0;
  } else {
    ok = ok && fputs("# Begin: Data Text\n", F.f) >= 0;
    std::string row;
    for (int64_t c = 0; ok && c < n3 / 3; ++c) {
      row = num(m_aos[3 * c]) + " " + num(m_aos[3 * c + 1]) + " " + num(m_aos[3 * c + 2]) + "\n";
      ok = fwrite(row.data(), 1, row.size(), F.f) == row.size();
    }
    ok = ok && fputs("# End: Data Text\n", F.f) >= 0;
  }
  ok = ok && fputs("# End: Segment\n", F.f) >= 0;
  if (!ok) return err(MM_ERR_ARG, "write to " + fn + " failed");
  FILE* f = F.f;
  F.f = nullptr;
  if (fclose(f) != 0) return err(MM_ERR_ARG, "close of " + fn + " failed");
  return MM_OK;
}

int mm_ovf_read_header(const char* path, mm_mesh_desc* mesh, int* type, char* title, size_t title_cap) {
  if (!path || !mesh) return err(MM_ERR_ARG, "mm_ovf_read_header: null argument");
  const std::string fn = with_ext(path);
  File F;
  F.f = fopen(fn.c_str(), "rb");
  if (!F.f) return err(MM_ERR_ARG, "cannot open " + fn + ": " + std::strerror(errno));
  Header h;
  if (int rc = read_header(F.f, h)) return rc;
  mesh->nx = static_cast<int>(h.nx);
  mesh->ny = static_cast<int>(h.ny);
  mesh->nz = static_cast<int>(h.nz);
  mesh->dx = h.dx;
  mesh->dy = h.dy;
  mesh->dz = h.dz;
  mesh->pbc = 0;
  if (type) *type = h.type;
  if (title && title_cap > 0) {
    const size_t n = std::min(title_cap - 1, h.title.size());
    std::memcpy(title, h.title.data(), n);
    title[n] = '\0';
  }
  return MM_OK;
}

// data of read_ovf(fname)  src/ovf2.jl:210-291, as float64
int mm_ovf_read(const char* path, double* m_aos, int64_t ncells) {
  if (!path || !m_aos) return err(MM_ERR_ARG, "mm_ovf_read: null argument");
  const std::string fn = with_ext(path);
  File F;
  F.f = fopen(fn.c_str(), "rb");
  if (!F.f) return err(MM_ERR_ARG, "cannot open " + fn + ": " + std::strerror(errno));
  Header h;
  if (int rc = read_header(F.f, h)) return rc;
  if (h.nx * h.ny * h.nz != ncells) return err(MM_ERR_ARG, "The ovf does not match the sim.mesh");
  return read_data(F.f, h, m_aos);
}

}  // extern "C"
