/* Protobuf binary wire format for the two gsbn messages read or written as
 * files: StimRawData (stimulus tables, ProcExtGen.cpp:61-89) and SolverState
 * (snapshots, Database.cpp:257-295, Solver.cpp:45-62), field numbers from
 * src/gsbn/proto/gsbn.proto.
 *
 * A reader of tagged fields: varint (wire type 0), fixed64 (1),
 * length-delimited (2), fixed32 (5).  Repeated scalars are accepted packed
 * (one length-delimited run) or one tag per element, as protobuf parsers
 * accept both; unknown fields are skipped by wire type; a missing required
 * field, a truncated buffer or a wrong wire type for a known field is an
 * error.  The writer emits packed repeated fields (the schema's [packed=true]
 * fields) and fields in number order, as protobuf serialisers do.
 */
#include <cstring>
#include <fstream>
#include <sstream>

#include "gsbn_engine.hpp"

namespace gsbn {

namespace {

class Reader {
 public:
  Reader(const uint8_t* p, size_t n, const char* what) : p_(p), e_(p + n), what_(what) {}
  bool done() const { return p_ >= e_; }

  uint64_t varint() {
    uint64_t v = 0;
    for (int s = 0; s < 64; s += 7) {
      if (p_ >= e_) bad("truncated varint");
      uint8_t b = *p_++;
      v |= (uint64_t)(b & 0x7f) << s;
      if (!(b & 0x80)) return v;
    }
    bad("varint longer than 10 bytes");
  }
  uint32_t fixed32() {
    if (e_ - p_ < 4) bad("truncated fixed32");
    uint32_t v;
    std::memcpy(&v, p_, 4);
    p_ += 4;
    return v;
  }
  uint64_t fixed64() {
    if (e_ - p_ < 8) bad("truncated fixed64");
    uint64_t v;
    std::memcpy(&v, p_, 8);
    p_ += 8;
    return v;
  }
  Reader sub() {
    uint64_t n = varint();
    if ((uint64_t)(e_ - p_) < n) bad("truncated length-delimited field");
    Reader r(p_, (size_t)n, what_);
    p_ += n;
    return r;
  }
  std::string bytes() {
    Reader r = sub();
    return std::string((const char*)r.p_, (size_t)(r.e_ - r.p_));
  }
  void skip(int wt) {
    switch (wt) {
      case 0: varint(); break;
      case 1: fixed64(); break;
      case 2: sub(); break;
      case 5: fixed32(); break;
      default: bad("unsupported wire type " + std::to_string(wt));
    }
  }
  /* repeated varint scalar: packed or not */
  template <class T>
  void rep_varint(int wt, std::vector<T>& out) {
    if (wt == 2) {
      Reader r = sub();
      while (!r.done()) out.push_back((T)r.varint());
    } else if (wt == 0) {
      out.push_back((T)varint());
    } else {
      bad("wrong wire type for a varint field");
    }
  }
  void rep_float(int wt, std::vector<float>& out) {
    if (wt == 2) {
      Reader r = sub();
      if ((r.e_ - r.p_) % 4) bad("packed float run not a multiple of 4 bytes");
      while (!r.done()) out.push_back(bits_f(r.fixed32()));
    } else if (wt == 5) {
      out.push_back(bits_f(fixed32()));
    } else {
      bad("wrong wire type for a float field");
    }
  }
  void rep_double(int wt, std::vector<double>& out) {
    if (wt == 2) {
      Reader r = sub();
      if ((r.e_ - r.p_) % 8) bad("packed double run not a multiple of 8 bytes");
      while (!r.done()) {
        uint64_t u = r.fixed64();
        double d;
        std::memcpy(&d, &u, 8);
        out.push_back(d);
      }
    } else if (wt == 1) {
      uint64_t u = fixed64();
      double d;
      std::memcpy(&d, &u, 8);
      out.push_back(d);
    } else {
      bad("wrong wire type for a double field");
    }
  }
  float f32(int wt) {
    if (wt != 5) bad("wrong wire type for a float field");
    return bits_f(fixed32());
  }
  uint64_t u64(int wt) {
    if (wt != 0) bad("wrong wire type for an integer field");
    return varint();
  }
  static float bits_f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  }
  [[noreturn]] void bad(const std::string& m) const { fatal(std::string(what_) + ": " + m); }

 private:
  const uint8_t* p_;
  const uint8_t* e_;
  const char* what_;
};

void put_varint(std::string& o, uint64_t v) {
  while (v >= 0x80) {
    o.push_back((char)(v | 0x80));
    v >>= 7;
  }
  o.push_back((char)v);
}
void put_tag(std::string& o, int field, int wt) { put_varint(o, ((uint64_t)field << 3) | (uint64_t)wt); }
void put_f32(std::string& o, int field, float f) {
  put_tag(o, field, 5);
  char b[4];
  std::memcpy(b, &f, 4);
  o.append(b, 4);
}
void put_bytes(std::string& o, int field, const std::string& s) {
  put_tag(o, field, 2);
  put_varint(o, s.size());
  o += s;
}

std::string slurp(const std::string& path, const char* what) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fatal(std::string(what) + " file not found: " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return ss.str();
}

}  // namespace

StimRawData decode_stim_raw_data(const std::string& bytes) {
  StimRawData s;
  Reader r((const uint8_t*)bytes.data(), bytes.size(), "StimRawData");
  unsigned seen = 0;
  while (!r.done()) {
    uint64_t tag = r.varint();
    int field = (int)(tag >> 3), wt = (int)(tag & 7);
    switch (field) {
      case 1: s.data_rows = (uint32_t)r.u64(wt); seen |= 1; break;
      case 2: s.data_cols = (uint32_t)r.u64(wt); seen |= 2; break;
      case 3: r.rep_varint(wt, s.data); break;
      case 4: s.mask_rows = (uint32_t)r.u64(wt); seen |= 4; break;
      case 5: s.mask_cols = (uint32_t)r.u64(wt); seen |= 8; break;
      case 6: r.rep_float(wt, s.mask); break;
      default: r.skip(wt);
    }
  }
  if (seen != 15) r.bad("missing a required field (data_rows, data_cols, mask_rows, mask_cols)");
  /* ProcExtGen.cpp:80-88 */
  if (s.data.size() != (size_t)s.data_rows * s.data_cols) fatal("Bad stimuli: data size != data_rows*data_cols");
  if (s.mask.size() != (size_t)s.mask_rows * s.mask_cols) fatal("Bad stimuli: mask size != mask_rows*mask_cols");
  return s;
}

StimRawData read_stim_raw_data(const std::string& path) {
  return decode_stim_raw_data(slurp(path, "stimulus"));
}

/* ------------------------------------------------------------ SolverState */

void read_solver_state(const std::string& path, Database& db) {
  std::string buf = slurp(path, "snapshot");
  Reader r((const uint8_t*)buf.data(), buf.size(), "SolverState");
  unsigned seen = 0;
  while (!r.done()) {
    uint64_t tag = r.varint();
    int field = (int)(tag >> 3), wt = (int)(tag & 7);
    if (field == 1) {
      db.snapshot_timestamp = r.f32(wt);
      seen |= 1;
    } else if (field == 2) {
      db.snapshot_prn = r.f32(wt);
      seen |= 2;
    } else if (field >= 4 && field <= 10 && wt == 2) {
      /* VectorState{I8,I16,I32,I64,F16,F32,F64}: name 1, ld 2, data 3 */
      Reader v = r.sub();
      std::string name;
      std::vector<int64_t> ints;
      std::vector<float> floats;
      std::vector<double> doubles;
      while (!v.done()) {
        uint64_t t2 = v.varint();
        int f2 = (int)(t2 >> 3), w2 = (int)(t2 & 7);
        if (f2 == 1 && w2 == 2)
          name = v.bytes();
        else if (f2 == 3 && (field == 9 || field == 8))
          v.rep_float(w2, floats);
        else if (f2 == 3 && field == 10)
          v.rep_double(w2, doubles);
        else if (f2 == 3)
          v.rep_varint(w2, ints);
        else
          v.skip(w2);
      }
      Database::StateVec sv;
      if (field == 4) {
        sv.type = BCPNN_I8;
        sv.bytes.resize(ints.size());
        for (size_t i = 0; i < ints.size(); i++) sv.bytes[i] = (uint8_t)(int8_t)(int32_t)ints[i];
      } else if (field == 6) {
        sv.type = BCPNN_I32;
        sv.bytes.resize(ints.size() * 4);
        for (size_t i = 0; i < ints.size(); i++) {
          int32_t x = (int32_t)ints[i];
          std::memcpy(&sv.bytes[i * 4], &x, 4);
        }
      } else if (field == 9) {
        sv.type = BCPNN_F32;
        sv.bytes.resize(floats.size() * 4);
        if (!floats.empty()) std::memcpy(sv.bytes.data(), floats.data(), floats.size() * 4);
      } else {
        continue; /* i16/i64/f16/f64 vectors hold nothing of this path */
      }
      db.snapshot[name] = std::move(sv);
    } else {
      r.skip(wt);
    }
  }
  if ((seen & 3) != 3) r.bad("missing timestamp or prn");
}

std::string encode_solver_state(float timestamp, float prn,
                                const std::vector<std::pair<std::string, Database::StateVec>>& vecs) {
  std::string o;
  put_f32(o, 1, timestamp);
  put_f32(o, 2, prn);
  /* fields in number order: i8 (4), i32 (6), f32 (9) */
  for (int pass = 0; pass < 3; pass++) {
    int want = pass == 0 ? BCPNN_I8 : pass == 1 ? BCPNN_I32 : BCPNN_F32;
    int field = pass == 0 ? 4 : pass == 1 ? 6 : 9;
    for (auto& nv : vecs) {
      if (nv.second.type != want) continue;
      std::string m;
      put_bytes(m, 1, nv.first);
      std::string packed;
      const std::vector<uint8_t>& b = nv.second.bytes;
      if (want == BCPNN_I8) {
        for (uint8_t x : b) put_varint(packed, (uint64_t)(int64_t)(int8_t)x);
      } else if (want == BCPNN_I32) {
        for (size_t i = 0; i + 4 <= b.size(); i += 4) {
          int32_t x;
          std::memcpy(&x, &b[i], 4);
          put_varint(packed, (uint64_t)(int64_t)x);
        }
      } else {
        packed.assign((const char*)b.data(), b.size());
      }
      if (!packed.empty()) put_bytes(m, 3, packed);
      put_bytes(o, field, m);
    }
  }
  return o;
}

}  // namespace gsbn
