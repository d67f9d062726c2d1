// thx_checkpoint.cpp -- host-side checkpoint interchange in the reference's
// restart format, so that a state can move between this library and a
// reference run in either direction.
//
// Layout (src/Simulation.cpp:1560-1603, include/CheckpointConfig.hpp:75-92):
//   <dir>/Cycle<c>/checkpoint_cycle_<c>.<rank, 8 digits>.chk
//       "THESEUS_CHECKPOINT_RAW_V1\n", uint64 count, count raw doubles
//       (the rank's byNODES state vector, native byte order)
//   <dir>/Cycle<c>/checkpoint_cycle_<c>.json
//       the compatibility record of include/CheckpointConfig.hpp:94-111
// Loading follows src/Simulation.cpp:1477-1557 and the metadata checks of
// include/CheckpointConfig.hpp:113-172, with the same failure messages.
#include "theseus_b200.h"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

namespace {

const char kMagic[] = "THESEUS_CHECKPOINT_RAW_V1";

void set_msg(char *msg, size_t len, const std::string &text) {
  if (!msg || len == 0) return;
  std::snprintf(msg, len, "%s", text.c_str());
}

// ---- a minimal JSON reader: one object of scalars (nested values skipped) --

struct JValue {
  enum Kind { NUL, BOOL, NUM, STR, OTHER } kind = NUL;
  bool b = false;
  double num = 0.0;
  bool integral = false;
  long long i = 0;
  std::string s;
};

class JParser {
 public:
  explicit JParser(const char *p) : p_(p) {}
  bool object(std::map<std::string, JValue> &out) {
    ws();
    if (*p_ != '{') return false;
    ++p_;
    ws();
    if (*p_ == '}') { ++p_; return tail(); }
    for (;;) {
      ws();
      std::string key;
      if (!string(key)) return false;
      ws();
      if (*p_ != ':') return false;
      ++p_;
      JValue v;
      if (!value(v, 0)) return false;
      out[key] = v;
      ws();
      if (*p_ == ',') { ++p_; continue; }
      if (*p_ == '}') { ++p_; return tail(); }
      return false;
    }
  }

 private:
  bool tail() {
    ws();
    return *p_ == '\0';
  }
  void ws() {
    while (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r') ++p_;
  }
  bool string(std::string &s) {
    if (*p_ != '"') return false;
    ++p_;
    while (*p_ && *p_ != '"') {
      if (*p_ == '\\') {
        ++p_;
        switch (*p_) {
          case '"': s += '"'; break;
          case '\\': s += '\\'; break;
          case '/': s += '/'; break;
          case 'b': s += '\b'; break;
          case 'f': s += '\f'; break;
          case 'n': s += '\n'; break;
          case 'r': s += '\r'; break;
          case 't': s += '\t'; break;
          case 'u': {  // keep ASCII code points, replace the rest
            unsigned cp = 0;
            for (int k = 1; k <= 4; ++k) {
              const char c = p_[k];
              cp <<= 4;
              if (c >= '0' && c <= '9') cp |= (unsigned)(c - '0');
              else if (c >= 'a' && c <= 'f') cp |= (unsigned)(c - 'a' + 10);
              else if (c >= 'A' && c <= 'F') cp |= (unsigned)(c - 'A' + 10);
              else return false;
            }
            s += cp < 0x80 ? (char)cp : '?';
            p_ += 4;
            break;
          }
          default: return false;
        }
        ++p_;
      } else {
        s += *p_++;
      }
    }
    if (*p_ != '"') return false;
    ++p_;
    return true;
  }
  bool value(JValue &v, int depth) {
    ws();
    if (depth > 64) return false;
    const char c = *p_;
    if (c == '"') {
      v.kind = JValue::STR;
      return string(v.s);
    }
    if (c == '{' || c == '[') {  // skipped: only scalars are read
      v.kind = JValue::OTHER;
      const char close = c == '{' ? '}' : ']';
      ++p_;
      ws();
      if (*p_ == close) { ++p_; return true; }
      for (;;) {
        if (c == '{') {
          ws();
          std::string k;
          if (!string(k)) return false;
          ws();
          if (*p_ != ':') return false;
          ++p_;
        }
        JValue inner;
        if (!value(inner, depth + 1)) return false;
        ws();
        if (*p_ == ',') { ++p_; continue; }
        if (*p_ == close) { ++p_; return true; }
        return false;
      }
    }
    if (!std::strncmp(p_, "true", 4)) { v.kind = JValue::BOOL; v.b = true; p_ += 4; return true; }
    if (!std::strncmp(p_, "false", 5)) { v.kind = JValue::BOOL; v.b = false; p_ += 5; return true; }
    if (!std::strncmp(p_, "null", 4)) { v.kind = JValue::NUL; p_ += 4; return true; }
    if (c == '-' || (c >= '0' && c <= '9')) {
      const char *start = p_;
      bool frac = false;
      if (*p_ == '-') ++p_;
      while ((*p_ >= '0' && *p_ <= '9') || *p_ == '.' || *p_ == 'e' || *p_ == 'E' || *p_ == '+' ||
             *p_ == '-') {
        if (*p_ == '.' || *p_ == 'e' || *p_ == 'E') frac = true;
        ++p_;
      }
      const std::string tok(start, p_);
      char *end = nullptr;
      errno = 0;
      v.kind = JValue::NUM;
      v.num = std::strtod(tok.c_str(), &end);
      if (!end || *end != '\0') return false;
      if (!frac) {
        errno = 0;
        v.i = std::strtoll(tok.c_str(), &end, 10);
        v.integral = errno == 0 && end && *end == '\0';
      }
      return true;
    }
    return false;
  }
  const char *p_;
};

// shortest decimal that reads back to the same double
std::string fmt_double(double x) {
  char buf[40];
  for (int prec = 1; prec <= 17; ++prec) {
    std::snprintf(buf, sizeof(buf), "%.*g", prec, x);
    if (std::strtod(buf, nullptr) == x) break;
  }
  std::string s(buf);
  if (std::isfinite(x) && s.find_first_of(".eEn") == std::string::npos) s += ".0";
  return s;
}

std::string metadata_json(double time, int cycle, const thx_checkpoint_compat &c) {
  // keys in the order a sorted-key JSON object prints them, two-space indent
  std::ostringstream o;
  o << "{\n"
    << "  \"cycle\": " << cycle << ",\n"
    << "  \"dimension\": " << c.dimension << ",\n"
    << "  \"format_version\": 2,\n"
    << "  \"geometry\": \"" << (c.axisymmetric ? "axisymmetric" : "cartesian") << "\",\n"
    << "  \"global_dofs\": " << (long long)c.global_dofs << ",\n"
    << "  \"global_elements\": " << (long long)c.global_elements << ",\n"
    << "  \"mpi_ranks\": " << c.mpi_ranks << ",\n"
    << "  \"num_equations\": " << c.num_equations << ",\n"
    << "  \"order\": " << c.order << ",\n"
    << "  \"real_bytes\": " << c.real_bytes << ",\n"
    << "  \"state_format\": \"raw_vector_v1\",\n"
    << "  \"state_representation\": \"conservative\",\n"
    << "  \"time\": " << fmt_double(time) << "\n"
    << "}\n";
  return o.str();
}

std::filesystem::path cycle_dir(const char *dir, int cycle) {
  return std::filesystem::path(dir) / ("Cycle" + std::to_string(cycle));
}
std::filesystem::path metadata_file(const char *dir, int cycle) {
  return cycle_dir(dir, cycle) / ("checkpoint_cycle_" + std::to_string(cycle) + ".json");
}
std::filesystem::path rank_file(const char *dir, int cycle, int rank) {
  char name[96];
  std::snprintf(name, sizeof(name), "checkpoint_cycle_%d.%08d.chk", cycle, rank);
  return cycle_dir(dir, cycle) / name;
}

// include/CheckpointConfig.hpp:113-172; returns THX_OK and *current (false
// for legacy metadata) or THX_ERR_INVALID_ARGUMENT with the reason in msg.
int validate(const std::map<std::string, JValue> &m, const thx_checkpoint_compat &e, int *current,
             char *msg, size_t len) {
  auto str = [&](const char *k) -> std::string {
    auto it = m.find(k);
    return it != m.end() && it->second.kind == JValue::STR ? it->second.s : std::string();
  };
  auto fail = [&](const std::string &why) {
    set_msg(msg, len, why);
    return THX_ERR_INVALID_ARGUMENT;
  };
  auto fv = m.find("format_version");
  if (fv == m.end()) {
    if (e.axisymmetric) return fail("Legacy checkpoint cannot establish axisymmetric conservative-state semantics");
    *current = 0;
    return THX_OK;
  }
  if (fv->second.kind != JValue::NUM || !fv->second.integral || (fv->second.i != 1 && fv->second.i != 2))
    return fail("Unsupported checkpoint metadata format version");
  const long long version = fv->second.i;
  if (str("state_format") != "raw_vector_v1") return fail("Unsupported checkpoint state format");
  if (version == 1 && e.axisymmetric)
    return fail("Version 1 checkpoint cannot establish whether an axisymmetric state stores U or rU");
  if (version == 2) {
    if (str("state_representation") != "conservative")
      return fail("Unsupported checkpoint state representation");
    if (str("geometry") != (e.axisymmetric ? "axisymmetric" : "cartesian"))
      return fail("Checkpoint is incompatible with the current run: geometry differs");
  }
  auto num = [&](const char *k, long long *v) {
    auto it = m.find(k);
    if (it == m.end() || it->second.kind != JValue::NUM) return false;
    *v = it->second.integral ? it->second.i : (long long)it->second.num;
    return true;
  };
  long long rb = 0;
  if (!num("real_bytes", &rb) || rb != e.real_bytes)
    return fail("Checkpoint floating-point representation differs");
  const std::pair<const char *, long long> req[] = {
      {"mpi_ranks", e.mpi_ranks},           {"order", e.order},
      {"dimension", e.dimension},           {"num_equations", e.num_equations},
      {"global_elements", e.global_elements}, {"global_dofs", e.global_dofs}};
  for (const auto &r : req) {
    long long v = 0;
    if (!num(r.first, &v) || v != r.second)
      return fail(std::string("Checkpoint is incompatible with the current run: ") + r.first + " differs");
  }
  *current = 1;
  return THX_OK;
}

}  // namespace

extern "C" {

int thx_checkpoint_metadata(double time, int cycle, const thx_checkpoint_compat *c, char *buf,
                            size_t len) {
  if (!c || !buf) return THX_ERR_INVALID_ARGUMENT;
  const std::string s = metadata_json(time, cycle, *c);
  if (s.size() + 1 > len) return THX_ERR_INVALID_ARGUMENT;
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return THX_OK;
}

int thx_checkpoint_validate(const char *json, const thx_checkpoint_compat *expected, int *current_format,
                            char *msg, size_t msg_len) {
  if (!json || !expected || !current_format) return THX_ERR_INVALID_ARGUMENT;
  std::map<std::string, JValue> m;
  if (!JParser(json).object(m)) {
    set_msg(msg, msg_len, "Checkpoint metadata is not a JSON object");
    return THX_ERR_INVALID_ARGUMENT;
  }
  return validate(m, *expected, current_format, msg, msg_len);
}

int thx_checkpoint_save(const char *directory, int cycle, int rank, double time,
                        const thx_checkpoint_compat *compat, const double *state, int64_t count,
                        int write_metadata, char *msg, size_t msg_len) {
  if (!directory || !compat || (!state && count > 0) || count < 0 || rank < 0) return THX_ERR_INVALID_ARGUMENT;
  try {
    std::error_code ec;
    std::filesystem::create_directories(cycle_dir(directory, cycle), ec);
    if (ec) {
      set_msg(msg, msg_len, "Failed to create checkpoint directory " + cycle_dir(directory, cycle).string() +
                                ": " + ec.message());
      return THX_ERR_IO;
    }
    const auto rf = rank_file(directory, cycle, rank);
    {
      std::ofstream f(rf, std::ios::binary);
      if (!f) {
        set_msg(msg, msg_len, "Failed to open checkpoint state for writing: " + rf.string());
        return THX_ERR_IO;
      }
      const uint64_t n = (uint64_t)count;
      f << kMagic << "\n";
      f.write(reinterpret_cast<const char *>(&n), sizeof(n));
      f.write(reinterpret_cast<const char *>(state), (std::streamsize)(n * sizeof(double)));
      f.close();
      if (!f) {
        set_msg(msg, msg_len, "Failed while writing checkpoint state: " + rf.string());
        return THX_ERR_IO;
      }
    }
    if (write_metadata) {
      const auto mf = metadata_file(directory, cycle);
      std::ofstream f(mf);
      if (!f) {
        set_msg(msg, msg_len, "Failed to open checkpoint metadata for writing: " + mf.string());
        return THX_ERR_IO;
      }
      f << metadata_json(time, cycle, *compat);
      f.close();
      if (!f) {
        set_msg(msg, msg_len, "Failed while writing checkpoint metadata: " + mf.string());
        return THX_ERR_IO;
      }
    }
  } catch (const std::exception &ex) {
    set_msg(msg, msg_len, ex.what());
    return THX_ERR_IO;
  }
  return THX_OK;
}

int thx_checkpoint_load(const char *directory, int cycle, int rank, const thx_checkpoint_compat *expected,
                        double *time, double *state, int64_t count, char *msg, size_t msg_len) {
  if (!directory || !expected || !time || (!state && count > 0) || count < 0 || rank < 0)
    return THX_ERR_INVALID_ARGUMENT;
  try {
    const auto mf = metadata_file(directory, cycle);
    std::ifstream ms(mf);
    if (!ms) {
      set_msg(msg, msg_len, "Failed to open checkpoint metadata: " + mf.string());
      return THX_ERR_IO;
    }
    std::stringstream text;
    text << ms.rdbuf();
    std::map<std::string, JValue> m;
    if (!JParser(text.str().c_str()).object(m)) {
      set_msg(msg, msg_len, "Checkpoint metadata is not a JSON object: " + mf.string());
      return THX_ERR_INVALID_ARGUMENT;
    }
    auto cy = m.find("cycle");
    const long long stored = cy != m.end() && cy->second.kind == JValue::NUM ? (long long)cy->second.num : 0;
    if (stored != cycle) {
      set_msg(msg, msg_len, "Checkpoint cycle mismatch: requested " + std::to_string(cycle) +
                                " but metadata contains " + std::to_string(stored));
      return THX_ERR_INVALID_ARGUMENT;
    }
    auto tm = m.find("time");
    if (tm == m.end() || tm->second.kind != JValue::NUM) {
      set_msg(msg, msg_len, "Checkpoint metadata does not contain a simulation time");
      return THX_ERR_INVALID_ARGUMENT;
    }
    int current = 0;
    int st = validate(m, *expected, &current, msg, msg_len);
    if (st) return st;
    if (!current) {
      set_msg(msg, msg_len, "Legacy checkpoints store an MFEM grid function, which is not read here");
      return THX_ERR_UNSUPPORTED;
    }
    const auto rf = rank_file(directory, cycle, rank);
    std::ifstream f(rf, std::ios::binary);
    if (!f) {
      set_msg(msg, msg_len, "Failed to open checkpoint state for reading: " + rf.string());
      return THX_ERR_IO;
    }
    std::string magic;
    std::getline(f, magic);
    if (magic != kMagic) {
      set_msg(msg, msg_len, "Invalid checkpoint state header in " + rf.string());
      return THX_ERR_INVALID_ARGUMENT;
    }
    uint64_t n = 0;
    f.read(reinterpret_cast<char *>(&n), sizeof(n));
    if (!f || n != (uint64_t)count) {
      set_msg(msg, msg_len, "Checkpoint state size " + std::to_string(n) +
                                " does not match current finite-element space size " + std::to_string(count));
      return THX_ERR_INVALID_ARGUMENT;
    }
    f.read(reinterpret_cast<char *>(state), (std::streamsize)(n * sizeof(double)));
    if (!f) {
      set_msg(msg, msg_len, "Failed while reading checkpoint state: " + rf.string());
      return THX_ERR_IO;
    }
    *time = tm->second.num;
  } catch (const std::exception &ex) {
    set_msg(msg, msg_len, ex.what());
    return THX_ERR_IO;
  }
  return THX_OK;
}

}  // extern "C"
