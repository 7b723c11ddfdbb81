/* Protobuf text format reader for gsbn's SolverParam (src/gsbn/proto/gsbn.proto)
 * and the argument Parser (src/gsbn/Parser.cpp:12-43).
 *
 * Two stages: a tokenizer + recursive-descent parser that turns the text into
 * a generic tree of named fields (scalars kept as their token text), then a
 * binder per message type that checks every field against the schema
 * (name, scalar kind, label) and converts the values.  Number conversion
 * follows protobuf's text parser: floats are read as double (strtod) and
 * rounded once to float; integer fields take integer tokens only (decimal,
 * 0x hex or 0-prefixed octal) and are range-checked; "inf"/"nan" are
 * accepted for floats; adjacent string literals concatenate.
 */
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>

#include "gsbn_engine.hpp"

namespace gsbn {

void fatal(const std::string& msg) { throw Fatal(msg); }

namespace {

enum class Tok { End, Ident, Int, Float, String, Symbol };

struct Token {
  Tok kind = Tok::End;
  std::string text;
  int line = 0;
};

class Lexer {
 public:
  explicit Lexer(const std::string& s) : s_(s) { next(); }
  const Token& peek() const { return cur_; }
  Token take() {
    Token t = cur_;
    next();
    return t;
  }

 private:
  void skip_space() {
    for (;;) {
      while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\r' || s_[i_] == '\n' ||
                                s_[i_] == '\f' || s_[i_] == '\v')) {
        if (s_[i_] == '\n') line_++;
        i_++;
      }
      if (i_ < s_.size() && s_[i_] == '#') {
        while (i_ < s_.size() && s_[i_] != '\n') i_++;
        continue;
      }
      return;
    }
  }
  static bool ident_start(char c) { return (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '_'; }
  static bool ident_char(char c) { return ident_start(c) || (c >= '0' && c <= '9'); }
  static bool digit(char c) { return c >= '0' && c <= '9'; }

  void next() {
    skip_space();
    cur_ = Token();
    cur_.line = line_;
    if (i_ >= s_.size()) return;
    char c = s_[i_];
    if (ident_start(c)) {
      size_t b = i_;
      while (i_ < s_.size() && ident_char(s_[i_])) i_++;
      cur_.kind = Tok::Ident;
      cur_.text = s_.substr(b, i_ - b);
      return;
    }
    if (digit(c) || (c == '.' && i_ + 1 < s_.size() && digit(s_[i_ + 1]))) {
      size_t b = i_;
      bool is_float = false;
      if (c == '0' && i_ + 1 < s_.size() && (s_[i_ + 1] == 'x' || s_[i_ + 1] == 'X')) {
        i_ += 2;
        while (i_ < s_.size() && std::isxdigit((unsigned char)s_[i_])) i_++;
      } else {
        while (i_ < s_.size() && digit(s_[i_])) i_++;
        if (i_ < s_.size() && s_[i_] == '.') {
          is_float = true;
          i_++;
          while (i_ < s_.size() && digit(s_[i_])) i_++;
        }
        if (i_ < s_.size() && (s_[i_] == 'e' || s_[i_] == 'E')) {
          size_t save = i_;
          i_++;
          if (i_ < s_.size() && (s_[i_] == '+' || s_[i_] == '-')) i_++;
          if (i_ < s_.size() && digit(s_[i_])) {
            is_float = true;
            while (i_ < s_.size() && digit(s_[i_])) i_++;
          } else {
            i_ = save;
          }
        }
        if (i_ < s_.size() && (s_[i_] == 'f' || s_[i_] == 'F')) {
          is_float = true;
          i_++;
        }
      }
      if (i_ < s_.size() && ident_char(s_[i_]))
        fatal("line " + std::to_string(line_) + ": malformed number near '" + s_.substr(b, i_ - b + 1) + "'");
      cur_.kind = is_float ? Tok::Float : Tok::Int;
      cur_.text = s_.substr(b, i_ - b);
      return;
    }
    if (c == '"' || c == '\'') {
      cur_.kind = Tok::String;
      cur_.text = read_string(c);
      return;
    }
    cur_.kind = Tok::Symbol;
    cur_.text = std::string(1, c);
    i_++;
  }

  std::string read_string(char q) {
    std::string out;
    i_++;
    for (;;) {
      if (i_ >= s_.size() || s_[i_] == '\n') fatal("line " + std::to_string(line_) + ": unterminated string");
      char c = s_[i_++];
      if (c == q) break;
      if (c != '\\') {
        out.push_back(c);
        continue;
      }
      if (i_ >= s_.size()) fatal("line " + std::to_string(line_) + ": bad escape");
      char e = s_[i_++];
      switch (e) {
        case 'n': out.push_back('\n'); break;
        case 't': out.push_back('\t'); break;
        case 'r': out.push_back('\r'); break;
        case 'a': out.push_back('\a'); break;
        case 'b': out.push_back('\b'); break;
        case 'f': out.push_back('\f'); break;
        case 'v': out.push_back('\v'); break;
        case '\\': out.push_back('\\'); break;
        case '\'': out.push_back('\''); break;
        case '"': out.push_back('"'); break;
        case '?': out.push_back('?'); break;
        case 'x':
        case 'X': {
          int v = 0, n = 0;
          while (n < 2 && i_ < s_.size() && std::isxdigit((unsigned char)s_[i_])) {
            char h = s_[i_++];
            v = v * 16 + (digit(h) ? h - '0' : (std::tolower(h) - 'a' + 10));
            n++;
          }
          if (!n) fatal("line " + std::to_string(line_) + ": bad \\x escape");
          out.push_back((char)v);
          break;
        }
        default:
          if (e >= '0' && e <= '7') {
            int v = e - '0', n = 1;
            while (n < 3 && i_ < s_.size() && s_[i_] >= '0' && s_[i_] <= '7') {
              v = v * 8 + (s_[i_++] - '0');
              n++;
            }
            out.push_back((char)v);
          } else {
            fatal("line " + std::to_string(line_) + ": unknown escape \\" + std::string(1, e));
          }
      }
    }
    return out;
  }

  const std::string& s_;
  size_t i_ = 0;
  int line_ = 1;
  Token cur_;
};

/* generic tree */
struct Node;
struct Field {
  std::string name;
  int line = 0;
  bool is_msg = false;
  Token value;           /* scalar: Int/Float/String/Ident, text with a '-' prefix if negated */
  bool negative = false;
  std::shared_ptr<Node> msg;
};
struct Node {
  std::vector<Field> fields;
};

class TreeParser {
 public:
  explicit TreeParser(const std::string& text) : lx_(text) {}
  std::shared_ptr<Node> parse_top() {
    auto n = std::make_shared<Node>();
    parse_fields(*n, "");
    if (lx_.peek().kind != Tok::End) fatal(where() + "unexpected '" + lx_.peek().text + "'");
    return n;
  }

 private:
  std::string where() const { return "line " + std::to_string(lx_.peek().line) + ": "; }
  bool sym(const char* s) const { return lx_.peek().kind == Tok::Symbol && lx_.peek().text == s; }
  void expect(const char* s) {
    if (!sym(s)) fatal(where() + "expected '" + s + "', got '" + lx_.peek().text + "'");
    lx_.take();
  }

  void parse_fields(Node& n, const char* close) {
    for (;;) {
      const Token& t = lx_.peek();
      if (t.kind == Tok::End) {
        if (*close) fatal(where() + "missing '" + close + "'");
        return;
      }
      if (*close && sym(close)) return;
      if (t.kind != Tok::Ident) fatal(where() + "expected a field name, got '" + t.text + "'");
      Token name = lx_.take();
      bool colon = false;
      if (sym(":")) {
        lx_.take();
        colon = true;
      }
      if (sym("[")) {
        if (!colon) fatal(where() + "expected ':' before '['");
        lx_.take();
        if (!sym("]")) {
          for (;;) {
            parse_value(n, name);
            if (sym(",")) {
              lx_.take();
              continue;
            }
            break;
          }
        }
        expect("]");
      } else {
        if (!colon && !sym("{") && !sym("<")) fatal(where() + "expected ':' after " + name.text);
        parse_value(n, name);
      }
      if (sym(";") || sym(",")) lx_.take();
    }
  }

  void parse_value(Node& n, const Token& name) {
    Field f;
    f.name = name.text;
    f.line = name.line;
    if (sym("{") || sym("<")) {
      const char* close = sym("{") ? "}" : ">";
      lx_.take();
      f.is_msg = true;
      f.msg = std::make_shared<Node>();
      parse_fields(*f.msg, close);
      expect(close);
    } else {
      if (sym("-")) {
        lx_.take();
        f.negative = true;
      }
      const Token& t = lx_.peek();
      if (t.kind == Tok::String) {
        if (f.negative) fatal(where() + "'-' before a string");
        f.value = lx_.take();
        while (lx_.peek().kind == Tok::String) f.value.text += lx_.take().text;
      } else if (t.kind == Tok::Int || t.kind == Tok::Float || t.kind == Tok::Ident) {
        f.value = lx_.take();
      } else {
        fatal(where() + "expected a value for " + name.text);
      }
    }
    n.fields.push_back(std::move(f));
  }

  Lexer lx_;
};

/* ------------------------------------------------------------- binder */

class Bind {
 public:
  Bind(const Node& n, const char* type) : n_(n), type_(type) {}

  ~Bind() noexcept(false) {
    if (std::uncaught_exceptions()) return;
    for (const Field& f : n_.fields)
      if (!known_.count(f.name))
        fatal("line " + std::to_string(f.line) + ": message " + type_ + " has no field \"" + f.name + "\"");
  }

  template <class F>
  void each(const char* name, F fn) {
    known_.insert(name);
    for (const Field& f : n_.fields)
      if (f.name == name) fn(f);
  }

  /* optional/required scalar or message: at most once */
  const Field* one(const char* name, bool required) {
    known_.insert(name);
    const Field* got = nullptr;
    for (const Field& f : n_.fields) {
      if (f.name != name) continue;
      if (got)
        fatal("line " + std::to_string(f.line) + ": non-repeated field \"" + name + "\" of " + type_ +
              " given more than once");
      got = &f;
    }
    if (!got && required) fatal(std::string("message ") + type_ + " is missing required field \"" + name + "\"");
    return got;
  }

  void f32(const char* name, float& out, bool required) {
    if (const Field* f = one(name, required)) out = to_f32(*f);
  }
  void u32(const char* name, uint32_t& out, bool required) {
    if (const Field* f = one(name, required)) out = (uint32_t)to_int(*f, 0, 4294967295LL);
  }
  void i32(const char* name, int32_t& out, bool required) {
    if (const Field* f = one(name, required)) out = (int32_t)to_int(*f, INT32_MIN, INT32_MAX);
  }
  void str(const char* name, std::string& out, bool required) {
    if (const Field* f = one(name, required)) out = to_str(*f);
  }
  const Node* msg(const char* name, bool required) {
    const Field* f = one(name, required);
    if (!f) return nullptr;
    if (!f->is_msg) fatal("line " + std::to_string(f->line) + ": field \"" + name + "\" is a message");
    return f->msg.get();
  }

  static std::string loc(const Field& f) { return "line " + std::to_string(f.line) + ": "; }

  static float to_f32(const Field& f) {
    if (f.is_msg) fatal(loc(f) + "field \"" + f.name + "\" takes a number");
    double v;
    const std::string& t = f.value.text;
    if (f.value.kind == Tok::Ident) {
      std::string l;
      for (char c : t) l.push_back((char)std::tolower((unsigned char)c));
      if (l == "inf" || l == "infinity")
        v = INFINITY;
      else if (l == "nan")
        v = NAN;
      else
        fatal(loc(f) + "\"" + t + "\" is not a number");
    } else if (f.value.kind == Tok::Int) {
      v = (double)to_int(f, INT64_MIN / 2, INT64_MAX / 2, true);
      return (float)v;
    } else if (f.value.kind == Tok::Float) {
      std::string s = t;
      if (!s.empty() && (s.back() == 'f' || s.back() == 'F')) s.pop_back();
      errno = 0;
      char* end = nullptr;
      v = std::strtod(s.c_str(), &end);
      if (end == s.c_str() || *end) fatal(loc(f) + "bad number \"" + t + "\"");
    } else {
      fatal(loc(f) + "field \"" + f.name + "\" takes a number");
    }
    if (f.negative) v = -v;
    return (float)v;
  }

  static long long to_int(const Field& f, long long lo, long long hi, bool raw = false) {
    if (f.is_msg || f.value.kind != Tok::Int) fatal(loc(f) + "field \"" + f.name + "\" takes an integer");
    const std::string& t = f.value.text;
    int base = 10;
    const char* p = t.c_str();
    if (t.size() > 1 && t[0] == '0' && (t[1] == 'x' || t[1] == 'X')) {
      base = 16;
      p += 2;
    } else if (t.size() > 1 && t[0] == '0') {
      base = 8;
      p += 1;
    }
    errno = 0;
    char* end = nullptr;
    unsigned long long u = std::strtoull(p, &end, base);
    if (*end || errno == ERANGE || u > (unsigned long long)INT64_MAX) fatal(loc(f) + "bad integer \"" + t + "\"");
    long long v = (long long)u;
    if (f.negative) v = -v;
    if (!raw && (v < lo || v > hi)) fatal(loc(f) + "integer " + (f.negative ? "-" : "") + t + " out of range for " + f.name);
    return v;
  }

  static std::string to_str(const Field& f) {
    if (f.is_msg || f.value.kind != Tok::String) fatal(loc(f) + "field \"" + f.name + "\" takes a string");
    return f.value.text;
  }

 private:
  const Node& n_;
  const char* type_;
  std::set<std::string> known_;
};

ModeParam bind_mode(const Node& n) {
  ModeParam m;
  Bind b(n, "ModeParam");
  b.f32("begin_time", m.begin_time, true);
  b.f32("end_time", m.end_time, true);
  b.u32("begin_lgidx_id", m.begin_lgidx_id, false);
  b.u32("begin_lgexp_id", m.begin_lgexp_id, false);
  b.u32("begin_wmask_id", m.begin_wmask_id, false);
  b.u32("time_step", m.time_step, false);
  b.u32("lgidx_step", m.lgidx_step, false);
  b.u32("lgexp_step", m.lgexp_step, false);
  b.u32("wmask_step", m.wmask_step, false);
  b.f32("prn", m.prn, false);
  b.u32("plasticity", m.plasticity, false);
  return m;
}

GenParam bind_gen(const Node& n) {
  GenParam g;
  Bind b(n, "GenParam");
  b.str("stim_file", g.stim_file, false);
  b.f32("dt", g.dt, true);
  b.f32("eps", g.eps, true);
  b.each("mode_param", [&](const Field& f) {
    if (!f.is_msg) fatal(Bind::loc(f) + "mode_param is a message");
    g.mode_param.push_back(bind_mode(*f.msg));
  });
  b.each("procedure", [&](const Field& f) { g.procedure.push_back(Bind::to_str(f)); });
  return g;
}

PopParam bind_pop(const Node& n) {
  PopParam p;
  Bind b(n, "PopParam");
  b.u32("pop_num", p.pop_num, true);
  b.u32("hcu_num", p.hcu_num, true);
  b.u32("mcu_num", p.mcu_num, true);
  b.u32("fanout_num", p.fanout_num, true);
  b.f32("taum", p.taum, false);
  b.f32("wtagain", p.wtagain, false);
  b.f32("maxfq", p.maxfq, false);
  b.f32("igain", p.igain, false);
  b.f32("wgain", p.wgain, false);
  b.f32("lgbias", p.lgbias, false);
  b.f32("snoise", p.snoise, false);
  b.f32("adgain", p.adgain, false);
  b.f32("taua", p.taua, false);
  b.each("position", [&](const Field& f) { p.position.push_back((int32_t)Bind::to_int(f, INT32_MIN, INT32_MAX)); });
  b.each("shape", [&](const Field& f) { p.shape.push_back((uint32_t)Bind::to_int(f, 0, 4294967295LL)); });
  b.u32("type", p.type, false);
  b.u32("rank", p.rank, false);
  return p;
}

ProjParam bind_proj(const Node& n) {
  ProjParam q;
  Bind b(n, "ProjParam");
  b.u32("src_pop", q.src_pop, true);
  b.u32("dest_pop", q.dest_pop, true);
  b.f32("tauzi", q.tauzi, true);
  b.f32("tauzj", q.tauzj, true);
  b.f32("taue", q.taue, true);
  b.f32("taup", q.taup, true);
  b.f32("maxfq", q.maxfq, false);
  b.f32("bgain", q.bgain, false);
  b.f32("wgain", q.wgain, false);
  if (const Field* f = b.one("tauepsc", false)) {
    q.has_tauepsc = true;
    q.tauepsc = Bind::to_f32(*f);
  }
  b.f32("slot_num", q.slot_num, true);
  b.f32("distance", q.distance, false);
  return q;
}

ProcParam bind_proc(const Node& n) {
  ProcParam p;
  Bind b(n, "ProcParam");
  b.str("name", p.name, true);
  auto kv = [](const Field& f, const char* type, std::string& key) -> const Node& {
    if (!f.is_msg) fatal(Bind::loc(f) + f.name + " is a message");
    const Node& m = *f.msg;
    (void)type;
    (void)key;
    return m;
  };
  b.each("argi", [&](const Field& f) {
    std::string key;
    const Node& m = kv(f, "ProcParamArgI", key);
    Bind a(m, "ProcParamArgI");
    int32_t v = 0;
    a.str("key", key, true);
    a.i32("val", v, true);
    p.argi.emplace_back(key, v);
  });
  b.each("argf", [&](const Field& f) {
    std::string key;
    const Node& m = kv(f, "ProcParamArgF", key);
    Bind a(m, "ProcParamArgF");
    float v = 0.f;
    a.str("key", key, true);
    a.f32("val", v, true);
    p.argf.emplace_back(key, v);
  });
  b.each("args", [&](const Field& f) {
    std::string key;
    const Node& m = kv(f, "ProcParamArgS", key);
    Bind a(m, "ProcParamArgS");
    std::string v;
    a.str("key", key, true);
    a.str("val", v, true);
    p.args.emplace_back(key, v);
  });
  return p;
}

std::string g_float(float v) {
  /* shortest text that reads back to the same float */
  char buf[64];
  for (int prec = 6; prec <= 9; prec++) {
    std::snprintf(buf, sizeof buf, "%.*g", prec, (double)v);
    if ((float)std::strtod(buf, nullptr) == v || std::isnan(v)) break;
  }
  return buf;
}

}  // namespace

SolverParam parse_solver_param_text(const std::string& text) {
  auto root = TreeParser(text).parse_top();
  SolverParam sp;
  Bind b(*root, "SolverParam");
  sp.gen_param = bind_gen(*b.msg("gen_param", true));
  const Node* net = b.msg("net_param", true);
  {
    Bind nb(*net, "NetParam");
    nb.each("pop_param", [&](const Field& f) {
      if (!f.is_msg) fatal(Bind::loc(f) + "pop_param is a message");
      sp.net_param.pop_param.push_back(bind_pop(*f.msg));
    });
    nb.each("proj_param", [&](const Field& f) {
      if (!f.is_msg) fatal(Bind::loc(f) + "proj_param is a message");
      sp.net_param.proj_param.push_back(bind_proj(*f.msg));
    });
  }
  const Node* rec = b.msg("rec_param", true);
  {
    Bind rb(*rec, "RecParam");
    rb.str("directory", sp.rec_param.directory, false);
  }
  b.each("proc_param", [&](const Field& f) {
    if (!f.is_msg) fatal(Bind::loc(f) + "proc_param is a message");
    sp.proc_param.push_back(bind_proc(*f.msg));
  });
  return sp;
}

SolverParam read_solver_param(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) fatal("cannot open network description " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  try {
    return parse_solver_param_text(ss.str());
  } catch (const Fatal& e) {
    fatal(path + ": " + e.what());
  }
}

std::string dump_solver_param(const SolverParam& sp) {
  std::ostringstream o;
  const GenParam& g = sp.gen_param;
  o << "gen.stim_file=" << g.stim_file << "\n"
    << "gen.dt=" << g_float(g.dt) << "\n"
    << "gen.eps=" << g_float(g.eps) << "\n";
  for (size_t i = 0; i < g.mode_param.size(); i++) {
    const ModeParam& m = g.mode_param[i];
    o << "mode[" << i << "]=" << g_float(m.begin_time) << "," << g_float(m.end_time) << "," << m.begin_lgidx_id << ","
      << m.begin_lgexp_id << "," << m.begin_wmask_id << "," << m.time_step << "," << m.lgidx_step << ","
      << m.lgexp_step << "," << m.wmask_step << "," << g_float(m.prn) << "," << m.plasticity << "\n";
  }
  for (size_t i = 0; i < g.procedure.size(); i++) o << "gen.procedure[" << i << "]=" << g.procedure[i] << "\n";
  for (size_t i = 0; i < sp.net_param.pop_param.size(); i++) {
    const PopParam& p = sp.net_param.pop_param[i];
    o << "pop[" << i << "]=" << p.pop_num << "," << p.hcu_num << "," << p.mcu_num << "," << p.fanout_num << ","
      << g_float(p.taum) << "," << g_float(p.wtagain) << "," << g_float(p.maxfq) << "," << g_float(p.igain) << ","
      << g_float(p.wgain) << "," << g_float(p.lgbias) << "," << g_float(p.snoise) << "," << g_float(p.adgain) << ","
      << g_float(p.taua) << "," << p.type << "," << p.rank << ",pos";
    for (int32_t v : p.position) o << ":" << v;
    o << ",shape";
    for (uint32_t v : p.shape) o << ":" << v;
    o << "\n";
  }
  for (size_t i = 0; i < sp.net_param.proj_param.size(); i++) {
    const ProjParam& q = sp.net_param.proj_param[i];
    o << "proj[" << i << "]=" << q.src_pop << "," << q.dest_pop << "," << g_float(q.tauzi) << "," << g_float(q.tauzj)
      << "," << g_float(q.taue) << "," << g_float(q.taup) << "," << g_float(q.maxfq) << "," << g_float(q.bgain) << ","
      << g_float(q.wgain) << "," << (q.has_tauepsc ? g_float(q.tauepsc) : std::string("-")) << ","
      << g_float(q.slot_num) << "," << g_float(q.distance) << "\n";
  }
  o << "rec.directory=" << sp.rec_param.directory << "\n";
  for (size_t i = 0; i < sp.proc_param.size(); i++) {
    const ProcParam& p = sp.proc_param[i];
    o << "proc[" << i << "]=" << p.name << "\n";
    for (auto& kv : p.argi) o << "proc[" << i << "].argi." << kv.first << "=" << kv.second << "\n";
    for (auto& kv : p.argf) o << "proc[" << i << "].argf." << kv.first << "=" << g_float(kv.second) << "\n";
    for (auto& kv : p.args) o << "proc[" << i << "].args." << kv.first << "=" << kv.second << "\n";
  }
  return o.str();
}

bool Parser::argi(const std::string& key, int& val) const {
  for (auto& kv : p_.argi)
    if (kv.first == key) {
      val = kv.second;
      return true;
    }
  return false;
}

bool Parser::argf(const std::string& key, float& val) const {
  for (auto& kv : p_.argf)
    if (kv.first == key) {
      val = kv.second;
      return true;
    }
  return false;
}

bool Parser::args(const std::string& key, std::string& val) const {
  for (auto& kv : p_.args)
    if (kv.first == key) {
      val = kv.second;
      return true;
    }
  return false;
}

}  // namespace gsbn
