// input.cpp -- input.yaml to a request descriptor on the host, in C++.
//
// The host pipeline of the reference (src/iDFT/iDFT.jl:24-40: YAML.load_file,
// iLST, geometry_system, setup_iDFT) restated so that a server can turn request
// text into an sdft_system_desc without a Julia or Python host:
//   * a YAML subset (block and flow mappings and sequences, plain and quoted
//     scalars, comments) with the number rules of YAML.jl: exponent literals such
//     as 1e-6 are floats;
//   * the molecular system (src/molecular_system/setup/setup_molsys.jl:48-75):
//     constants and Bjerrum length, topology parser, reactions, species, used
//     monomers, state families, configurations, bonds, max-distance matrices,
//     monomer properties and the protonation work dmuH, with the reference's
//     quirks (temperature and dielectric constant read from `constraints:`,
//     bookkeeping reactions zeroed, neutralisation partners' pSpecies);
//   * the bulk state (src/iLST/evaluation/objective/solver_bulkstate.jl:31-104):
//     the AndersonResidual driver of AndersonResidual.jl:27-138 on the residual
//     of residual_bulkstate.jl:26-35, whose two expensive steps are
//     sdft_bulk_eval (bulk.cpp); when that driver diverges, the same residual
//     is solved by undamped Picard steps with Anderson acceleration, exactly as
//     the Python host does;
//   * the 1D Cartesian slit (src/geometry/setup/create_cartesian.jl:66) and the
//     fixed (grafted) segments (determine_fixed.jl:1-29).
// The Python host (softdft_b200/host) is the same pipeline; the tests compare
// the two descriptors.
#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/softdft.h"

namespace {

struct InputError : std::runtime_error {
  int code;
  InputError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void fail(const std::string& m, int code = SDFT_ERR_ARG) { throw InputError(code, m); }

// ===========================================================================
// YAML subset
// ===========================================================================
struct Node {
  enum Kind { Null, Scalar, Map, Seq } kind = Null;
  std::string text;  // scalar text
  bool quoted = false;
  std::vector<std::pair<std::string, Node>> map;
  std::vector<Node> seq;

  const Node* get(const std::string& k) const {
    if (kind != Map) return nullptr;
    for (const auto& kv : map)
      if (kv.first == k) return &kv.second;
    return nullptr;
  }
  bool has(const std::string& k) const { return get(k) != nullptr; }
  // a repeated key keeps its first position and takes the last value, as
  // YAML.jl's and PyYAML's mapping constructors do
  void put(const std::string& k, Node v) {
    for (auto& kv : map)
      if (kv.first == k) {
        kv.second = std::move(v);
        return;
      }
    map.emplace_back(k, std::move(v));
  }
};

bool match_digits(const std::string& s, size_t& i, bool underscores) {
  const size_t b = i;
  while (i < s.size() && (std::isdigit((unsigned char)s[i]) || (underscores && i > b && s[i] == '_'))) i++;
  return i > b;
}

// YAML 1.1 ints (decimal) and the float forms of the reader (YAML 1.2 exponents included)
bool is_int_text(const std::string& s) {
  size_t i = 0;
  if (i < s.size() && (s[i] == '+' || s[i] == '-')) i++;
  return match_digits(s, i, true) && i == s.size();
}
bool is_float_text(const std::string& s) {
  static const char* specials[] = {".inf", ".Inf", ".INF", "+.inf", "+.Inf", "+.INF", "-.inf", "-.Inf", "-.INF",
                                   ".nan", ".NaN", ".NAN"};
  for (const char* sp : specials)
    if (s == sp) return true;
  size_t i = 0;
  if (i < s.size() && (s[i] == '+' || s[i] == '-')) i++;
  bool digits = match_digits(s, i, true);
  bool dot = false;
  if (i < s.size() && s[i] == '.') {
    dot = true;
    i++;
    bool frac = match_digits(s, i, true);
    if (!digits && !frac) return false;
    if (!digits && (s[0] == '+' || s[0] == '-')) return false;  // "-.5" is not a float in the reader
  } else if (!digits) {
    return false;
  }
  if (i < s.size() && (s[i] == 'e' || s[i] == 'E')) {
    i++;
    if (i < s.size() && (s[i] == '+' || s[i] == '-')) i++;
    if (!match_digits(s, i, false)) return false;
  } else if (!dot) {
    return false;
  }
  return i == s.size();
}
bool is_bool_text(const std::string& s, bool* v) {
  static const char* t[] = {"true", "True", "TRUE", "yes", "Yes", "YES", "on", "On", "ON"};
  static const char* f[] = {"false", "False", "FALSE", "no", "No", "NO", "off", "Off", "OFF"};
  for (const char* x : t)
    if (s == x) return *v = true, true;
  for (const char* x : f)
    if (s == x) return *v = false, true;
  return false;
}
double parse_number(std::string s) {
  s.erase(std::remove(s.begin(), s.end(), '_'), s.end());
  if (s == ".inf" || s == ".Inf" || s == ".INF" || s == "+.inf" || s == "+.Inf" || s == "+.INF") return INFINITY;
  if (s == "-.inf" || s == "-.Inf" || s == "-.INF") return -INFINITY;
  if (s == ".nan" || s == ".NaN" || s == ".NAN") return NAN;
  // strtod keeps an underflow (subnormal or zero) and an overflow (infinity),
  // as parse(Float64, s) does
  const char* b = s.c_str();
  char* e = nullptr;
  const double v = std::strtod(b, &e);
  if (s.empty() || std::isspace((unsigned char)s[0]) || e != b + s.size()) fail("not a number: " + s);
  return v;
}

// Float64(v) for numbers, parse(Float64, string(v)) otherwise (process_numerical.jl:17-28)
double as_float(const Node& n) {
  if (n.kind != Node::Scalar) fail("expected a number");
  bool b;
  if (!n.quoted && is_bool_text(n.text, &b)) return b ? 1.0 : 0.0;
  try {
    return parse_number(n.text);
  } catch (const InputError&) {
    throw;
  } catch (...) {
    fail("not a number: " + n.text);
  }
}
bool is_float_node(const Node& n) { return n.kind == Node::Scalar && !n.quoted && is_float_text(n.text); }
int as_int(const Node& n) {
  const double v = as_float(n);
  if (!(v == std::floor(v)) || v < INT32_MIN || v > INT32_MAX) fail("not an integer: " + n.text);
  return (int)v;
}
// Python truthiness of the loaded value (bool(entry.get(key, False)))
bool truthy(const Node* n) {
  if (!n || n->kind == Node::Null) return false;
  if (n->kind != Node::Scalar) return n->kind == Node::Map ? !n->map.empty() : !n->seq.empty();
  bool b;
  if (!n->quoted && is_bool_text(n->text, &b)) return b;
  if (!n->quoted && (is_int_text(n->text) || is_float_text(n->text))) return parse_number(n->text) != 0.0;
  return !n->text.empty();
}
// the entries a `for x in v` loop visits in Julia: a sequence's items, or a
// scalar itself
std::vector<Node> listed(const Node& n) {
  if (n.kind == Node::Seq) return n.seq;
  if (n.kind == Node::Scalar) return {n};
  fail("expected a list");
}
std::string as_str(const Node& n) {
  if (n.kind != Node::Scalar) fail("expected a scalar");
  return n.text;
}

struct Line {
  int indent;
  std::string text;
  int number;
};

std::string strip_comment(const std::string& s) {
  char q = 0;
  for (size_t i = 0; i < s.size(); i++) {
    const char c = s[i];
    if (q) {
      if (c == q) q = 0;
    } else if (c == '\'' || c == '"') {
      q = c;
    } else if (c == '#' && (i == 0 || std::isspace((unsigned char)s[i - 1]))) {
      return s.substr(0, i);
    }
  }
  return s;
}
std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) a++;
  while (b > a && std::isspace((unsigned char)s[b - 1])) b--;
  return s.substr(a, b - a);
}

Node make_scalar(const std::string& raw) {
  Node n;
  const std::string t = trim(raw);
  if (t.empty() || t == "~" || t == "null" || t == "Null" || t == "NULL") {
    n.kind = Node::Null;
    return n;
  }
  n.kind = Node::Scalar;
  if (t.size() >= 2 && (t[0] == '\'' || t[0] == '"') && t.back() == t[0]) {
    n.quoted = true;
    std::string body = t.substr(1, t.size() - 2);
    if (t[0] == '\'') {  // '' is a quote
      std::string o;
      for (size_t i = 0; i < body.size(); i++) {
        o += body[i];
        if (body[i] == '\'' && i + 1 < body.size() && body[i + 1] == '\'') i++;
      }
      body = o;
    } else {  // the common escapes
      std::string o;
      for (size_t i = 0; i < body.size(); i++) {
        if (body[i] == '\\' && i + 1 < body.size()) {
          const char e = body[++i];
          o += e == 'n' ? '\n' : e == 't' ? '\t' : e;
        } else {
          o += body[i];
        }
      }
      body = o;
    }
    n.text = body;
  } else {
    // YAML reserves these indicators at the start of a plain scalar (tags,
    // anchors, aliases, block scalars, directives, @ and `)
    if (std::strchr("!&*|>%@`", t[0])) fail("a plain scalar cannot start with '" + t.substr(0, 1) + "'");
    n.text = t;
  }
  return n;
}

// flow collections: [a, b], {k: v}, nested
struct Flow {
  const std::string& s;
  size_t i = 0;
  int line;
  void ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) i++;
  }
  Node value() {
    ws();
    if (i >= s.size()) fail("line " + std::to_string(line) + ": unexpected end of a flow collection");
    if (s[i] == '[') {
      i++;
      Node n;
      n.kind = Node::Seq;
      ws();
      if (i < s.size() && s[i] == ']') return i++, n;
      for (;;) {
        n.seq.push_back(value());
        ws();
        if (i < s.size() && s[i] == ',') {
          i++;
          ws();
          if (i < s.size() && s[i] == ']') return i++, n;
          continue;
        }
        if (i < s.size() && s[i] == ']') return i++, n;
        fail("line " + std::to_string(line) + ": expected , or ] in a flow sequence");
      }
    }
    if (s[i] == '{') {
      i++;
      Node n;
      n.kind = Node::Map;
      ws();
      if (i < s.size() && s[i] == '}') return i++, n;
      for (;;) {
        const std::string key = as_key(scalar_text(true));
        ws();
        if (i >= s.size() || s[i] != ':') fail("line " + std::to_string(line) + ": expected : in a flow mapping");
        i++;
        Node v = value_or_null();
        n.put(key, std::move(v));
        ws();
        if (i < s.size() && s[i] == ',') {
          i++;
          continue;
        }
        if (i < s.size() && s[i] == '}') return i++, n;
        fail("line " + std::to_string(line) + ": expected , or } in a flow mapping");
      }
    }
    return make_scalar(scalar_text(false));
  }
  Node value_or_null() {
    ws();
    if (i < s.size() && (s[i] == ',' || s[i] == '}')) return Node{};
    return value();
  }
  std::string scalar_text(bool key) {
    ws();
    const size_t b = i;
    if (i < s.size() && (s[i] == '\'' || s[i] == '"')) {
      const char q = s[i++];
      while (i < s.size()) {
        if (s[i] == q) {
          if (q == '\'' && i + 1 < s.size() && s[i + 1] == '\'') {
            i += 2;
            continue;
          }
          i++;
          break;
        }
        if (q == '"' && s[i] == '\\') i++;
        i++;
      }
      return s.substr(b, i - b);
    }
    while (i < s.size() && s[i] != ',' && s[i] != ']' && s[i] != '}' &&
           !(key && s[i] == ':' && (i + 1 >= s.size() || std::isspace((unsigned char)s[i + 1]) || s[i + 1] == ',')))
      i++;
    return s.substr(b, i - b);
  }
  static std::string as_key(const std::string& raw) {
    const Node k = make_scalar(raw);
    return k.kind == Node::Null ? std::string() : k.text;
  }
};

Node parse_inline(const std::string& text, int line) {
  const std::string t = trim(text);
  if (!t.empty() && (t[0] == '[' || t[0] == '{')) {
    Flow f{t, 0, line};
    Node n = f.value();
    f.ws();
    if (f.i != t.size()) fail("line " + std::to_string(line) + ": text after a flow collection");
    return n;
  }
  if (!t.empty() && (t[0] == '|' || t[0] == '>' || t[0] == '&' || t[0] == '*' || t[0] == '!'))
    fail("line " + std::to_string(line) + ": block scalars, anchors, aliases and tags are not supported");
  if (t == "-" || t.rfind("- ", 0) == 0) fail("line " + std::to_string(line) + ": a sequence entry after a key on its line");
  return make_scalar(t);
}

// position of the ': ' (or final ':') that separates a block mapping key from its value
size_t key_colon(const std::string& t) {
  // a block key is a quoted scalar or a plain scalar; inside a plain key,
  // brackets and quotes are ordinary characters.  A line that opens a flow
  // collection is a value (flow collections as keys are not read).
  if (!t.empty() && (t[0] == '[' || t[0] == '{')) return std::string::npos;
  size_t i = 0;
  if (!t.empty() && (t[0] == '\'' || t[0] == '"')) {
    const char q = t[0];
    for (i = 1; i < t.size(); i++) {
      if (q == '"' && t[i] == '\\') {
        i++;
      } else if (t[i] == q) {
        if (q == '\'' && i + 1 < t.size() && t[i + 1] == '\'') {
          i++;  // '' inside a single-quoted scalar
        } else {
          break;
        }
      }
    }
    if (i >= t.size()) return std::string::npos;
  }
  for (; i < t.size(); i++)
    if (t[i] == ':' && (i + 1 == t.size() || t[i + 1] == ' ' || t[i + 1] == '\t')) return i;
  return std::string::npos;
}

struct Block {
  std::vector<Line> L;
  size_t i = 0;

  Node parse(int indent) {
    if (i >= L.size()) return Node{};
    if (L[i].text == "-" || L[i].text.rfind("- ", 0) == 0) return seq(indent);
    return mapping(indent);
  }
  Node seq(int indent) {
    Node n;
    n.kind = Node::Seq;
    while (i < L.size() && L[i].indent == indent && (L[i].text == "-" || L[i].text.rfind("- ", 0) == 0)) {
      std::string rest = L[i].text.size() > 1 ? L[i].text.substr(2) : std::string();
      size_t pad = 0;
      while (pad < rest.size() && rest[pad] == ' ') pad++;
      rest = rest.substr(pad);
      const int col = indent + 2 + (int)pad;
      if (rest.empty()) {
        i++;
        if (i < L.size() && L[i].indent > indent) n.seq.push_back(parse(L[i].indent));
        else n.seq.push_back(Node{});
      } else if (rest == "-" || rest.rfind("- ", 0) == 0 || key_colon(rest) != std::string::npos) {
        // a nested sequence or mapping that starts on the item's line
        L[i].indent = col;
        L[i].text = rest;
        n.seq.push_back(parse(col));
      } else {
        n.seq.push_back(parse_inline(rest, L[i].number));
        i++;
      }
    }
    return n;
  }
  Node mapping(int indent) {
    Node n;
    n.kind = Node::Map;
    while (i < L.size() && L[i].indent == indent) {
      const std::string& t = L[i].text;
      if (t == "-" || t.rfind("- ", 0) == 0) fail("line " + std::to_string(L[i].number) + ": sequence item inside a mapping");
      const size_t c = key_colon(t);
      if (c == std::string::npos) fail("line " + std::to_string(L[i].number) + ": expected 'key: value'");
      const std::string key = Flow::as_key(t.substr(0, c));
      const std::string val = trim(t.substr(c + 1));
      const int ln = L[i].number;
      i++;
      Node v;
      if (!val.empty()) {
        v = parse_inline(val, ln);
      } else if (i < L.size() && L[i].indent > indent) {
        v = parse(L[i].indent);
      } else if (i < L.size() && L[i].indent == indent && (L[i].text == "-" || L[i].text.rfind("- ", 0) == 0)) {
        v = seq(indent);  // a sequence may sit at its key's indentation
      }
      n.put(key, std::move(v));
    }
    if (i < L.size() && L[i].indent > indent) fail("line " + std::to_string(L[i].number) + ": unexpected indentation");
    return n;
  }
};

// bracket depth a line leaves open (flow collections may span lines), counted
// from a flow collection that opens the line's value; brackets inside a plain
// scalar are text
int flow_depth(std::string t) {
  while (t == "-" || t.rfind("- ", 0) == 0) t = trim(t.substr(1));
  if (t.empty()) return 0;
  if (t[0] != '[' && t[0] != '{') {
    const size_t c = key_colon(t);
    if (c == std::string::npos) return 0;
    t = trim(t.substr(c + 1));
    if (t.empty() || (t[0] != '[' && t[0] != '{')) return 0;
  }
  int d = 0;
  char q = 0;
  for (char c : t) {
    if (q) {
      if (c == q) q = 0;
    } else if (c == '\'' || c == '"') {
      q = c;
    } else if (c == '[' || c == '{') {
      d++;
    } else if (c == ']' || c == '}') {
      d--;
    }
  }
  return d;
}

Node load_yaml(const std::string& text) {
  Block b;
  std::vector<std::string> raw;
  for (size_t pos = 0;;) {
    size_t e = text.find('\n', pos);
    if (e == std::string::npos) e = text.size();
    raw.push_back(text.substr(pos, e - pos));
    if (e == text.size()) break;
    pos = e + 1;
  }
  for (size_t k = 0; k < raw.size(); k++) {
    std::string line = raw[k];
    const int number = (int)k + 1;
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.find('\t') != std::string::npos && line.find_first_not_of(" \t") != std::string::npos &&
        line.find('\t') < line.find_first_not_of(" \t"))
      fail("line " + std::to_string(number) + ": tabs in indentation");
    line = strip_comment(line);
    std::string t = trim(line);
    if (t.empty() || t == "---" || t == "...") continue;
    if (line.rfind("%", 0) == 0) continue;  // directives (column 0 only)
    int ind = 0;
    while (ind < (int)line.size() && line[ind] == ' ') ind++;
    while (flow_depth(t) > 0 && k + 1 < raw.size()) {  // a flow collection continued on the next lines
      std::string next = raw[++k];
      if (!next.empty() && next.back() == '\r') next.pop_back();
      t += " " + trim(strip_comment(next));
    }
    b.L.push_back({ind, t, number});
  }
  if (b.L.empty()) fail("input.yaml is empty");
  Node root = b.parse(b.L[0].indent);
  if (b.i != b.L.size()) fail("line " + std::to_string(b.L[b.i].number) + ": unexpected indentation");
  if (root.kind != Node::Map) fail("input.yaml must hold a mapping at the top level");
  return root;
}

}  // namespace

namespace {

// ===========================================================================
// molecular system (src/molecular_system/setup/**)
// ===========================================================================
const double kLog10 = std::log(10.0);

struct Constants {  // structures/ConstantsStruct.jl:18-24 (SI)
  double epsilon0 = 8.854187817e-12, e0 = 1.60217653e-19, k_B = 1.3806505e-23, NA = 6.0221415e23, l_sc = 0.5e-9;
};
double concentration_to_density(double conc, const Constants& c) {  // conversions.jl:19-22
  const double vol_liters = std::pow(c.l_sc, 3.0) * 1000.0;
  return conc * c.NA * vol_liters;
}
double density_to_concentration(double rho, const Constants& c) {  // conversions.jl:8-12
  const double vol_liters = std::pow(c.l_sc, 3.0) * 1000.0;
  return rho / vol_liters / c.NA;
}

struct Topology {  // structures/TopologyStruct.jl:23-30, 0-based
  std::string monomers;
  std::vector<std::vector<int>> children, parents, levels;
};

// parse_topology.jl:16-127: letters, (group) and (group)k repeats; a letter's
// parent is the letter before it at the enclosing level.  A run of letters is
// walked iteratively (each letter one level deeper, child of the previous one);
// only parenthesised groups recurse, so long chains need no deep stack.
Topology parse_topology(const std::string& sequence) {
  std::vector<char> mons;
  std::vector<std::vector<int>> children, parents, levels;
  int current = 0;
  std::function<void(size_t, size_t, int, int, int)> rec = [&](size_t b, size_t e, int level, int parent, int depth) {
    if (depth > 256) fail("parenthesised groups nested too deeply");
    size_t i = b;
    while (i < e) {
      const char ch = sequence[i];
      if (std::isalpha((unsigned char)ch)) {
        const int cur = ++current;
        mons.push_back(ch);
        if (level > (int)levels.size()) levels.emplace_back();
        levels[level - 1].push_back(cur);
        if (parent == 0) {
          children.emplace_back();
          parents.emplace_back();
        } else {
          if (parent > (int)children.size()) children.push_back({cur});
          else children[parent - 1].push_back(cur);
          if (cur > (int)parents.size()) parents.push_back({parent});
          else parents[cur - 1].push_back(parent);
        }
        if (i + 1 >= e) children.emplace_back();  // the reference's trailing entry after a run's last letter
        parent = cur;
        level++;
        i++;
      } else if (ch == '(') {
        int bal = 1;
        size_t end = std::string::npos;
        for (size_t j2 = i + 1; j2 < e; j2++) {
          if (sequence[j2] == '(') bal++;
          else if (sequence[j2] == ')') bal--;
          if (bal == 0) {
            end = j2;
            break;
          }
        }
        if (end == std::string::npos) fail("Unmatched parenthesis in: " + sequence.substr(i, e - i));
        if (end == i + 1) fail("empty group in: " + sequence.substr(i, e - i));
        size_t k = end + 1;
        int mult = 1;
        if (k < e && std::isdigit((unsigned char)sequence[k])) {
          const size_t d0 = k;
          while (k < e && std::isdigit((unsigned char)sequence[k])) k++;
          if (k - d0 > 6) fail("group repeat count too large");
          mult = std::stoi(sequence.substr(d0, k - d0));
        }
        for (int r = 0; r < mult; r++) rec(i + 1, end, level, parent, depth + 1);
        i = k;  // the rest continues at this level from the same parent
      } else {
        fail(std::string("Not a recognized character: ") + ch);
      }
    }
  };
  if (sequence.empty()) fail("empty sequence");
  rec(0, sequence.size(), 1, 0, 0);
  Topology t;
  const int n = (int)mons.size();
  t.monomers.assign(mons.begin(), mons.end());
  for (int g = 0; g < n; g++) {
    std::vector<int> c;
    if (g < (int)children.size())
      for (int x : children[g]) c.push_back(x - 1);
    t.children.push_back(c);
    std::vector<int> p;
    if (g < (int)parents.size())
      for (int x : parents[g]) p.push_back(x - 1);
    t.parents.push_back(p);
  }
  for (const auto& l : levels) {
    std::vector<int> v;
    for (int x : l) v.push_back(x - 1);
    t.levels.push_back(v);
  }
  return t;
}

struct Reaction {  // structures/ReactionStruct.jl:24-28
  std::vector<std::string> species;
  std::vector<int> coeffs;
  double pK;
  bool bookkeeping() const {
    for (int c : coeffs)
      if (c != 0) return false;
    return true;
  }
  void split(std::vector<std::string>& reac, std::vector<std::string>& prod) const {
    reac.clear();
    prod.clear();
    for (size_t k = 0; k < species.size(); k++) {
      if (coeffs[k] == -1) reac.push_back(species[k]);
      else if (coeffs[k] == 1) prod.push_back(species[k]);
    }
  }
};

struct SpeciesEntry {  // parse_species.jl:29-36
  std::string name, role;
  double density, concentration, pSpecies;
  bool adjustable;
};

struct Config {  // structures/ConfigurationStruct.jl:41-47
  std::string model;
  std::vector<int> sequence, states;
  Topology topo;
  std::vector<std::vector<int>> family;
  std::vector<double> max_distance;  // n*n row-major when set
};

struct MolSys {
  Constants c;
  double bjerrum = 0.0;
  std::vector<std::string> fe_model, species, monomers;
  std::map<std::string, int> used;
  std::map<std::string, std::vector<std::string>> families;
  std::vector<Reaction> reactions;
  std::vector<Config> configs;
  std::vector<std::pair<int, int>> bonds;
  std::vector<double> diameters, valences, dmu, densities, pS, charge;
  std::vector<char> adjustable, compensator;
};

std::vector<Reaction> parse_reactions(const Node& ds) {  // parse_reactions.jl:30-73
  std::vector<Reaction> out;
  const Node* raw = ds.get("reactions");
  if (!raw || raw->kind == Node::Null) return out;
  if (raw->kind != Node::Seq) fail("Expected 'reactions' to be a list of reaction entries");
  for (const Node& r : raw->seq) {
    const Node* sp = r.get("species");
    const Node* cf = r.get("coeffs");
    const Node* pk = r.get("pK");
    if (!sp || !cf || !pk || sp->kind != Node::Seq || cf->kind != Node::Seq) fail("reaction needs species, coeffs and pK");
    if (sp->seq.size() != cf->seq.size()) fail("Mismatch between number of species and coefficients in a reaction");
    Reaction x;
    for (const Node& s : sp->seq) x.species.push_back(as_str(s));
    for (const Node& c : cf->seq) {
      const double v = as_float(c);
      const int ci = (int)std::nearbyint(v);
      if (std::fabs(v - ci) > 1e-8) fail("Non-integer stoichiometric coefficient in a reaction");
      if (ci != 1 && ci != -1) fail("Unsupported coefficient " + std::to_string(ci) + " in a reaction");
      x.coeffs.push_back(ci);
    }
    x.pK = as_float(*pk);
    out.push_back(x);
  }
  return out;
}

std::vector<SpeciesEntry> parse_species(const Node& ds) {  // parse_species.jl:38-82
  const Node* sps = ds.get("species");
  if (!sps || sps->kind != Node::Seq) fail("Input file is missing the required 'species' section.");
  std::vector<SpeciesEntry> out;
  for (const Node& e : sps->seq) {
    const Node* seq = e.get("sequence");
    if (!seq) fail("Each species must define a 'sequence' field.");
    SpeciesEntry s;
    s.name = as_str(*seq);
    const bool hd = e.has("density"), hc = e.has("concentration"), hp = e.has("pSpecies");
    s.adjustable = truthy(e.get("adjustable"));
    s.role = e.has("role") ? as_str(*e.get("role")) : std::string("monomer");
    if ((hd || hc) && hp)
      fail("Species '" + s.name + "' is overspecified: both 'density/concentration' and 'pSpecies' are defined.");
    if (hd && hc) fail("Species '" + s.name + "' is overspecified: both 'density' and 'concentration'.");
    if (hp && s.adjustable) fail("Species '" + s.name + "' has 'pSpecies' and is also marked as 'adjustable'.");
    s.density = hd ? as_float(*e.get("density")) : 0.0;
    s.concentration = hc ? as_float(*e.get("concentration")) : 0.0;
    s.pSpecies = hp ? as_float(*e.get("pSpecies")) : NAN;
    out.push_back(s);
  }
  return out;
}

std::set<std::string> neutralization_participants(const std::vector<Reaction>& rx) {  // state_families.jl:213-231
  std::set<std::string> out;
  std::vector<std::string> reac, prod;
  for (const Reaction& r : rx) {
    r.split(reac, prod);
    if (reac.empty() || prod.empty())
      for (const auto& s : reac.empty() ? prod : reac) out.insert(s);
  }
  return out;
}

using Graph = std::map<std::string, std::set<std::string>>;
std::set<std::string> component(const Graph& nb, const std::string& start) {
  std::set<std::string> seen;
  std::vector<std::string> stack{start};
  while (!stack.empty()) {
    const std::string n = stack.back();
    stack.pop_back();
    if (seen.count(n)) continue;
    seen.insert(n);
    auto it = nb.find(n);
    if (it != nb.end())
      for (const auto& m : it->second) stack.push_back(m);
  }
  return seen;
}

// connected components of the monomer graph induced by reactions (state_families.jl:1-166)
std::map<std::string, std::vector<std::string>> build_state_families(std::vector<SpeciesEntry>& entries,
                                                                     const std::vector<Reaction>& rx) {
  const auto neutral = neutralization_participants(rx);
  for (auto& e : entries)
    if (neutral.count(e.name)) e.role = "neutralizer";
  std::map<std::string, std::string> roles;
  for (const auto& e : entries) roles[e.name] = e.role;
  auto role = [&](const std::string& s) {
    auto it = roles.find(s);
    return it == roles.end() ? std::string("monomer") : it->second;
  };
  std::set<std::string> polymer;
  for (const auto& e : entries)
    if (e.name.size() > 1)
      for (char ch : e.name)
        if (std::isalpha((unsigned char)ch)) polymer.insert(std::string(1, ch));
  Graph nb;
  std::vector<std::pair<std::vector<std::string>, std::vector<std::string>>> pending;
  std::vector<std::string> reac, prod;
  for (const Reaction& r : rx) {
    r.split(reac, prod);
    if (reac.empty() || prod.empty()) {
      for (const auto& s : reac.empty() ? prod : reac)
        if (polymer.count(s))
          fail("Monomer '" + s + "' appears in a neutralization reaction, but it is part of a polymer sequence.");
      continue;
    }
    const size_t nr = reac.size(), np = prod.size();
    if (!((nr == 1 && (np == 1 || np == 2)) || (nr == 2 && np == 1))) fail("Unsupported reaction form");
    if (nr == 2 && np == 1 && role(reac[0]) == "monomer" && role(reac[1]) == "monomer")
      fail("Reaction has two reactants and one product, but both reactants are :monomer.");
    if (nr == 1 && np == 2 && role(prod[0]) == "monomer" && role(prod[1]) == "monomer")
      fail("Reaction has one reactant and two products, but both products are :monomer.");
    std::vector<std::string> lhs, rhs;
    for (const auto& s : reac)
      if (role(s) != "partner" && role(s) != "neutralizer") lhs.push_back(s);
    for (const auto& s : prod)
      if (role(s) != "partner" && role(s) != "neutralizer") rhs.push_back(s);
    const size_t tot = lhs.size() + rhs.size();
    if (tot > 2) fail("Reaction connects more than two candidate monomers.");
    if (tot == 2) {
      if (lhs.empty() || rhs.empty()) fail("Reaction: candidate monomers on one side only.");
      nb[lhs[0]].insert(rhs[0]);
      nb[rhs[0]].insert(lhs[0]);
    } else if (tot == 1) {
      pending.emplace_back(reac, prod);
    }
  }
  for (const auto& pr : pending) {  // resolve_pending_edges! (state_families.jl:93-125)
    std::vector<std::string> all = pr.first, cands;
    all.insert(all.end(), pr.second.begin(), pr.second.end());
    std::vector<std::string> uniq;
    for (const auto& s : all)
      if (std::find(uniq.begin(), uniq.end(), s) == uniq.end()) uniq.push_back(s);
    for (const auto& s : uniq)
      if (roles.count(s) && roles[s] == "monomer") cands.push_back(s);
    if (cands.size() != 2) continue;
    const std::string a = cands[0], b = cands[1];
    const auto fa = component(nb, a), fb = component(nb, b);
    nb[a];
    nb[b];
    if (fb.count(a) || fa.count(b)) continue;
    nb[a].insert(b);
    nb[b].insert(a);
  }
  std::set<std::string> all_mon;
  for (const auto& e : entries)
    for (char ch : e.name)
      if (std::isalpha((unsigned char)ch)) all_mon.insert(std::string(1, ch));
  std::map<std::string, std::vector<std::string>> families;
  std::set<std::string> visited;
  for (const auto& mon : all_mon) {
    if (visited.count(mon)) continue;
    std::vector<std::string> group;
    for (const auto& m : component(nb, mon))
      if (!visited.count(m)) {
        visited.insert(m);
        group.push_back(m);
      }
    std::sort(group.begin(), group.end());
    for (const auto& m : group) families[m] = group;
  }
  return families;
}

// bidirectional BFS path lengths, bond length (d_i + d_j)/2 (freely_jointed.jl:45-113)
std::vector<double> max_distance_matrix(const Config& cfg, const std::vector<double>& diam) {
  const int n = (int)cfg.sequence.size();
  std::vector<double> mat((size_t)n * n, 0.0);
  for (int start = 0; start < n; start++) {
    std::vector<double> dist(n, 0.0);
    std::vector<std::pair<int, double>> queue{{start, 0.0}};
    std::vector<char> visited(n, 0);
    visited[start] = 1;
    size_t head = 0;
    while (head < queue.size()) {
      const int cur = queue[head].first;
      const double d = queue[head].second;
      head++;
      std::vector<int> nbs = cfg.topo.children[cur];
      nbs.insert(nbs.end(), cfg.topo.parents[cur].begin(), cfg.topo.parents[cur].end());
      for (int nb : nbs) {
        if (nb < n && !visited[nb]) {
          const double dij = (diam[cfg.sequence[cur]] + diam[cfg.sequence[nb]]) / 2.0;
          const double nd = d + dij;
          dist[nb] = std::max(dist[nb], nd);
          queue.emplace_back(nb, nd);
          visited[nb] = 1;
        }
      }
    }
    for (int j = 0; j < n; j++) mat[(size_t)start * n + j] = dist[j];
  }
  for (int i = 0; i < n; i++) mat[(size_t)i * n + i] = 0.0;
  return mat;
}

// ideal protonation work relative to each family's alphabetically first member
// (assign_delta_muH.jl:50-248); mutates pS and zeroes resolved reactions
std::vector<double> assign_delta_muH(const std::vector<double>* valences, const std::map<std::string, int>& used,
                                     const std::map<std::string, std::vector<std::string>>& families,
                                     std::vector<Reaction>& rx, const std::vector<std::string>& names,
                                     const std::vector<double>& densities, std::vector<double>& pS, const Constants& c) {
  std::map<std::string, int> name_to_index;  // a repeated name maps to its last entry, as a Julia Dict does
  for (size_t i = 0; i < names.size(); i++) name_to_index[names[i]] = (int)i;
  auto idx_of = [&](const std::string& s) {
    auto it = name_to_index.find(s);
    if (it == name_to_index.end()) fail("species " + s + " is not defined in the species list");
    return it->second;
  };
  std::vector<double> delta(used.size(), 0.0);
  std::vector<std::string> reac, prod;
  for (const Reaction& r : rx) {  // step 1: neutralisation partners
    r.split(reac, prod);
    if (reac.empty() || prod.empty()) {
      const auto& side = reac.empty() ? prod : reac;
      if (side.size() != 2) fail("a neutralisation reaction needs two species on one side");
      const double dmu_total = -kLog10 * r.pK;
      const int i1 = idx_of(side[0]), i2 = idx_of(side[1]);
      const double p1 = pS[i1], p2 = pS[i2];
      if (!std::isnan(p1)) {
        const double d1 = -kLog10 * p1;
        pS[i2] = (dmu_total - d1) / -kLog10;
      } else if (!std::isnan(p2)) {
        const double d2 = -kLog10 * p2;
        pS[i1] = (dmu_total - d2) / -kLog10;
      }
    }
  }
  std::vector<std::pair<std::string, std::vector<std::pair<std::string, double>>>> graph;  // insertion order
  auto adj = [&](const std::string& m) -> std::vector<std::pair<std::string, double>>& {
    for (auto& kv : graph)
      if (kv.first == m) return kv.second;
    graph.emplace_back(m, std::vector<std::pair<std::string, double>>());
    return graph.back().second;
  };
  for (Reaction& r : rx) {  // step 2: the dmu graph
    r.split(reac, prod);
    if (valences) {
      double dq = 0.0;
      for (size_t k = 0; k < r.species.size(); k++) {
        auto it = used.find(r.species[k]);
        if (it != used.end()) dq += r.coeffs[k] * (*valences)[it->second];
      }
      if (std::fabs(dq) > 1e-6) fail("A reaction violates charge neutrality");
    }
    std::vector<std::string> sr, spd;
    for (const auto& s : reac)
      if (families.count(s)) sr.push_back(s);
    for (const auto& s : prod)
      if (families.count(s)) spd.push_back(s);
    bool found = false;
    std::string mon1, mon2;
    std::vector<std::string> fam1;
    for (const auto& a : sr) {
      for (const auto& b : spd) {
        mon1 = a;
        mon2 = b;
        fam1 = families.at(mon1);
        if (families.at(mon1) == families.at(mon2)) {
          found = true;
          break;
        }
      }
      if (found) break;
    }
    if (!found) continue;
    std::vector<std::string> sorted_fam = fam1;
    std::sort(sorted_fam.begin(), sorted_fam.end());
    const std::string base = sorted_fam[0];
    const bool fwd = mon1 == base;
    const std::string frm = fwd ? mon1 : mon2, to = fwd ? mon2 : mon1;
    double dmu = kLog10 * r.pK;
    for (size_t k = 0; k < r.species.size(); k++) {
      const std::string& sp = r.species[k];
      const int cf = r.coeffs[k];
      if (sp == mon1 || sp == mon2) continue;
      auto it = name_to_index.find(sp);
      if (it == name_to_index.end()) fail("Context species " + sp + " is not defined in species list.");
      const double ps = pS[it->second];
      if (!std::isnan(ps)) {
        dmu -= kLog10 * ps * cf;
      } else {
        const double rho = densities[it->second];
        if (rho > 0) {
          const double conc = density_to_concentration(rho, c);
          dmu += cf * -std::log(conc);
        } else {
          dmu = 0.0;
        }
      }
    }
    adj(frm).emplace_back(to, dmu);
    adj(to).emplace_back(frm, dmu);
    std::fill(r.coeffs.begin(), r.coeffs.end(), 0);
  }
  for (const auto& kv : families) {  // step 3: from each family's base along the graph
    std::vector<std::string> fam = kv.second;
    std::sort(fam.begin(), fam.end());
    const std::string base = fam[0];
    std::vector<std::pair<std::string, double>> work{{base, 0.0}};
    std::set<std::string> visited;
    std::function<void(const std::string&, double)> dfs = [&](const std::string& mon, double acc) {
      visited.insert(mon);
      for (const auto& e : adj(mon))
        if (!visited.count(e.first)) {
          bool set = false;
          for (auto& w : work)
            if (w.first == e.first) w.second = acc + e.second, set = true;
          if (!set) work.emplace_back(e.first, acc + e.second);
          dfs(e.first, acc + e.second);
        }
    };
    dfs(base, 0.0);
    for (const auto& w : work) delta[used.at(w.first)] = w.second;
    delta[used.at(base)] = 0.0;
  }
  for (Reaction& r : rx) {  // step 4: neutralisation with a defined pSpecies becomes bookkeeping
    r.split(reac, prod);
    bool nonzero = true;
    for (int cf : r.coeffs) nonzero &= cf != 0;
    if ((reac.empty() || prod.empty()) && nonzero) {
      const auto& side = reac.empty() ? prod : reac;
      const double p1 = pS[idx_of(side[0])], p2 = pS[idx_of(side[1])];
      if (!std::isnan(p1) || !std::isnan(p2)) std::fill(r.coeffs.begin(), r.coeffs.end(), 0);
    }
  }
  return delta;
}

// setup_molsys.jl:48-75
MolSys molecular_system(const Node& ds) {
  MolSys m;
  if (const Node* ru = ds.get("reduced_units"))  // process_constants.jl:10-16 (l_sc in nm)
    if (const Node* l = ru->get("l_sc")) m.c.l_sc = as_float(*l) * 1e-9;
  // temperature and dielectric constant come from `constraints:` and must be
  // Float64 values (get_temperature.jl:14-21, get_dielectric_constant.jl:15-22)
  auto constraint = [&](const char* key, double dflt) {
    const Node* cons = ds.get("constraints");
    const Node* v = cons ? cons->get(key) : nullptr;
    if (!v) return dflt;
    if (!is_float_node(*v)) fail(std::string(key) + " must be a Float64 value.");
    return as_float(*v);
  };
  const double T = constraint("temperature", 298.15), er = constraint("dielectric_constant", 78.4);
  m.bjerrum = std::pow(m.c.e0, 2.0) / (4 * M_PI * m.c.epsilon0 * er * m.c.k_B * T) / m.c.l_sc;
  const Node* model = ds.get("model");
  if (!model) fail("Input file is missing the required 'model' section.");
  if (model->kind == Node::Scalar) m.fe_model.push_back(model->text);
  else if (model->kind == Node::Seq)
    for (const Node& x : model->seq) m.fe_model.push_back(as_str(x));
  else fail("model must be a name or a list of names");
  m.reactions = parse_reactions(ds);
  auto entries = parse_species(ds);
  std::set<std::string> names_set;
  for (const auto& e : entries)
    for (char ch : e.name)
      if (std::isalpha((unsigned char)ch)) names_set.insert(std::string(1, ch));
  for (const auto& r : m.reactions)
    for (const auto& s : r.species) names_set.insert(s);
  int k = 0;
  for (const auto& s : names_set) {
    m.used[s] = k++;
    m.monomers.push_back(s);
  }
  m.families = build_state_families(entries, m.reactions);
  const Node& sps = *ds.get("species");
  for (const Node& s : sps.seq) {
    m.species.push_back(as_str(*s.get("sequence")));
    if (s.has("concentration")) m.densities.push_back(concentration_to_density(as_float(*s.get("concentration")), m.c));
    else m.densities.push_back(s.has("density") ? as_float(*s.get("density")) : 0.0);
    m.pS.push_back(s.has("pSpecies") ? as_float(*s.get("pSpecies")) : NAN);
    m.adjustable.push_back(truthy(s.get("adjustable")) ? 1 : 0);
  }
  m.compensator = m.adjustable;
  for (const Node& s : sps.seq) {  // process_configs.jl:25-83
    Config cfg;
    cfg.topo = parse_topology(as_str(*s.get("sequence")));
    cfg.model = s.has("model") ? as_str(*s.get("model")) : std::string("freely_jointed");
    if (cfg.model != "freely_jointed" && cfg.model != "monomerbead") fail("Unknown chain model " + cfg.model + ".");
    for (char ch : cfg.topo.monomers) {
      const std::string mon(1, ch);
      auto it = m.used.find(mon);
      if (it == m.used.end()) fail("Monomer " + mon + " not found in used_monomers.");
      cfg.sequence.push_back(it->second);
      auto f = m.families.find(mon);
      std::vector<int> idxs;
      if (f != m.families.end())
        for (const auto& x : f->second) idxs.push_back(m.used.at(x));
      else idxs.push_back(it->second);
      cfg.states.push_back((int)idxs.size());
      cfg.family.push_back(idxs);
    }
    m.configs.push_back(cfg);
  }
  std::set<std::pair<int, int>> bonds;  // process_bonds.jl:8-29
  for (const Config& cfg : m.configs)
    for (const auto& level : cfg.topo.levels)
      for (int child : level)
        for (int j : cfg.family[child])
          for (int parent : cfg.topo.parents[child])
            for (int j1 : cfg.family[parent]) bonds.insert({std::min(j, j1), std::max(j, j1)});
  m.bonds.assign(bonds.begin(), bonds.end());
  // process_monomers.jl:35-70: scalar properties pluralised, zero where unset
  const size_t nb = m.used.size();
  std::map<std::string, std::vector<double>> props;
  const Node* mdata = ds.get("monomers");
  for (const auto& name : m.monomers) {
    const Node* md = mdata ? mdata->get(name) : nullptr;
    if (!md) fail("Species " + name + " listed in used_monomers not found in dataset[\"monomers\"]");
    if (md->kind != Node::Map) fail("the properties of monomer " + name + " must be a mapping");
    for (const auto& kv : md->map) {
      if (kv.second.kind == Node::Map) continue;
      auto& v = props[kv.first + "s"];
      if (v.empty()) v.assign(nb, 0.0);
      v[m.used.at(name)] = as_float(kv.second);
    }
  }
  const std::vector<double>* val = props.count("valences") ? &props["valences"] : nullptr;
  m.dmu = assign_delta_muH(val, m.used, m.families, m.reactions, m.species, m.densities, m.pS, m.c);
  m.valences = val ? *val : std::vector<double>(nb, 0.0);
  if (props.count("diameters")) m.diameters = props["diameters"];
  m.charge.assign(m.configs.size(), 0.0);
  if (val)  // assign_species_charge.jl:1-20
    for (size_t u = 0; u < m.configs.size(); u++) {
      double q = 0.0;
      for (int b : m.configs[u].sequence) q += m.valences[b];
      m.charge[u] = q;
    }
  for (Config& cfg : m.configs)  // process_bonding.jl:12-16 (the matrices are built where used: grafted species)
    if (cfg.model == "freely_jointed" && m.diameters.empty())
      fail("Missing 'diameters' in properties.monomers. This is required for freely_jointed species_model.");
  if (m.diameters.empty()) m.diameters.assign(nb, 0.0);
  return m;
}

}  // namespace

namespace {

// ===========================================================================
// bulk state (src/iLST/**)
// ===========================================================================
struct Bulk {
  std::vector<double> rho_species, rho_beads, rho_bonds, mu_species, mu_ex, lng, Xi, segs;
  int iterations = 0;
  double residual = 0.0;
};

// numpy's pairwise summation of a contiguous float64 array (the reduction the
// Python host's np.sum performs), so that the two hosts sum in the same order
double np_sum(const double* a, size_t n) {
  if (n < 8) {
    double r = 0.0;
    for (size_t i = 0; i < n; i++) r += a[i];
    return r;
  }
  if (n <= 128) {
    double r[8];
    for (int j = 0; j < 8; j++) r[j] = a[j];
    size_t i = 8;
    for (; i < n - (n % 8); i += 8)
      for (int j = 0; j < 8; j++) r[j] += a[i + j];
    double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; i++) res += a[i];
    return res;
  }
  size_t n2 = n / 2;
  n2 -= n2 % 8;
  return np_sum(a, n2) + np_sum(a + n2, n - n2);
}

// the molecular system in the form sdft_bulk_eval takes
struct BulkSys {
  sdft_bulk_system sys{};
  std::vector<sdft_bulk_species> sp;
  std::vector<std::vector<int32_t>> ints;
  std::vector<int32_t> bond_types;
  size_t seg_total = 0;
};

const int32_t* keep_ints(BulkSys& b, std::vector<int32_t> v) {
  if (v.empty()) v.push_back(0);
  b.ints.push_back(std::move(v));
  return b.ints.back().data();
}

void build_bulk_sys(const MolSys& m, BulkSys& b) {
  uint32_t models = 0;  // bulk_chemical_potential.jl:9-25
  for (const auto& f : m.fe_model) {
    if (f == "ideal") models |= SDFT_BULK_IDEAL;
    else if (f == "mfmt") models |= SDFT_BULK_MFMT;
    else if (f == "TPT1mfmt") models |= SDFT_BULK_TPT1MFMT;
    else if (f == "msa") models |= SDFT_BULK_MSA;
    else if (f == "TPT1msa") models |= SDFT_BULK_TPT1MSA;
    else if (f != "coul") fail("Unknown or unsupported model(s): " + f, SDFT_ERR_UNSUPPORTED);
  }
  b.ints.reserve(8 * m.configs.size() + 1);
  b.sp.resize(m.configs.size());
  b.seg_total = 0;
  for (size_t u = 0; u < m.configs.size(); u++) {
    const Config& cfg = m.configs[u];
    const int n = (int)cfg.sequence.size();
    int S = 1, C = 1;
    for (const auto& f : cfg.family) S = std::max(S, (int)f.size());
    for (const auto& c : cfg.topo.children) C = std::max(C, (int)c.size());
    std::vector<int32_t> nst, states((size_t)n * S, -1), parent, nch, children((size_t)n * C, -1), lptr{0}, lsegs;
    for (int g = 0; g < n; g++) {
      nst.push_back((int)cfg.family[g].size());
      for (size_t i = 0; i < cfg.family[g].size(); i++) states[(size_t)g * S + i] = cfg.family[g][i];
      parent.push_back(cfg.topo.parents[g].empty() ? -1 : cfg.topo.parents[g][0]);
      nch.push_back((int)cfg.topo.children[g].size());
      for (size_t i = 0; i < cfg.topo.children[g].size(); i++) children[(size_t)g * C + i] = cfg.topo.children[g][i];
    }
    for (const auto& l : cfg.topo.levels) {
      lptr.push_back(lptr.back() + (int)l.size());
      lsegs.insert(lsegs.end(), l.begin(), l.end());
    }
    sdft_bulk_species& s = b.sp[u];
    s.n_seg = n;
    s.max_states = S;
    s.max_children = C;
    s.n_levels = (int)cfg.topo.levels.size();
    s.monomerbead = cfg.model == "monomerbead" ? 1 : 0;
    s.n_states = keep_ints(b, nst);
    s.states = keep_ints(b, states);
    s.parent = keep_ints(b, parent);
    s.n_children = keep_ints(b, nch);
    s.children = keep_ints(b, children);
    s.level_ptr = keep_ints(b, lptr);
    s.level_segs = keep_ints(b, lsegs);
    b.seg_total += (size_t)S * n;
  }
  for (const auto& bd : m.bonds) {
    b.bond_types.push_back(bd.first);
    b.bond_types.push_back(bd.second);
  }
  if (b.bond_types.empty()) b.bond_types.assign(2, 0);
  b.sys.nb = (int)m.monomers.size();
  b.sys.mb = (int)m.bonds.size();
  b.sys.ns = (int)m.configs.size();
  b.sys.models = models;
  b.sys.diameter = m.diameters.data();
  b.sys.valence = m.valences.data();
  b.sys.delta_muH = m.dmu.data();
  b.sys.bond_types = b.bond_types.data();
  b.sys.species = b.sp.data();
  b.sys.bjerrum_length = m.bjerrum;
}

int bond_index(const MolSys& m, int a, int b) {
  const std::pair<int, int> k{std::min(a, b), std::max(a, b)};
  for (size_t u = 0; u < m.bonds.size(); u++)
    if (m.bonds[u] == k) return (int)u;
  fail("bond missing from bond_types");
}

// initialize_densities.jl:31-121 (ideal state weights); also overwrites the
// species charge with the ideal state-averaged charge, as the reference does
Bulk initialize_densities(MolSys& m) {
  const size_t ns = m.species.size(), nb = m.monomers.size(), mb = m.bonds.size();
  Bulk b;
  b.rho_species.assign(ns, 0.0);
  b.rho_beads.assign(nb, 0.0);
  b.rho_bonds.assign(2 * mb, 0.0);
  b.mu_species.assign(ns, 0.0);
  b.mu_ex.assign(nb, 0.0);
  b.lng.assign(mb, 0.0);
  b.Xi.assign(ns, 0.0);
  const auto& dm = m.dmu;
  for (size_t u = 0; u < ns; u++) m.charge[u] = 0.0;
  for (size_t u = 0; u < m.configs.size(); u++) {
    const Config& cfg = m.configs[u];
    const int nseg = (int)cfg.sequence.size();
    const double dens = !std::isnan(m.pS[u]) ? concentration_to_density(std::pow(10.0, -m.pS[u]), m.c) : m.densities[u];
    const double pd = dens / nseg;
    b.rho_species[u] = pd;
    for (int si = 0; si < nseg; si++) {
      const auto& sti = cfg.family[si];
      double Qi = 0.0;
      for (int s : sti) Qi += std::exp(-dm[s]);
      for (int s_i : sti) {
        const double wi = std::exp(-dm[s_i]) / Qi;
        b.rho_beads[s_i] += pd * wi;
        m.charge[u] += wi * m.valences[s_i];
        if (!cfg.topo.parents[si].empty()) {
          const int sj = cfg.topo.parents[si][0];
          const auto& stj = cfg.family[sj];
          double Qj = 0.0;
          for (int s : stj) Qj += std::exp(-dm[s]);
          for (int s_j : stj) {
            const double wj = std::exp(-dm[s_j]) / Qj;
            const int bd = bond_index(m, s_i, s_j);
            b.rho_bonds[bd] += pd * wi * wj;
            b.rho_bonds[mb + bd] += pd * wi * wj;
          }
        }
      }
    }
  }
  return b;
}

std::set<std::string> species_in_reactions(const MolSys& m) {
  std::set<std::string> out;
  for (const auto& r : m.reactions)
    if (!r.bookkeeping()) out.insert(r.species.begin(), r.species.end());
  return out;
}

double sign_of(double x) { return x > 0 ? 1.0 : x < 0 ? -1.0 : 0.0; }

// balance_charge.jl:21-79 (strategy :equal)
void balance_charge(const MolSys& m, Bulk& b, double Q, std::vector<char>& adjustable) {
  const auto& sc = m.charge;
  if (Q == 0.0) {
    for (size_t i = 0; i < adjustable.size(); i++) adjustable[i] = m.compensator[i] && sign_of(sc[i]) == 1.0;
    return;
  }
  const double sQ = sign_of(Q);
  bool any = false;
  for (size_t i = 0; i < adjustable.size(); i++) {
    adjustable[i] = m.compensator[i] && sign_of(sc[i]) == -sQ;
    any |= adjustable[i] != 0;
  }
  if (!any) fail("No compensating species available to absorb net charge");
  double tw = 0.0;
  for (char a : adjustable) tw += a ? 1.0 : 0.0;
  for (size_t i = 0; i < adjustable.size(); i++) {
    if (adjustable[i]) {
      const double d = -Q * (1.0 / tw) / sc[i];
      b.rho_species[i] = m.densities[i] + std::max(d, 0.0);
    } else if (m.compensator[i]) {
      b.rho_species[i] = m.densities[i];
    }
  }
}

struct Residual {
  MolSys& m;
  BulkSys& bs;
  std::vector<int> rxn_species, ph_species;  // species whose log densities are unknowns, in order
  size_t n = 0;
  // assign_solution_variables (solver_bulkstate.jl:65-103)
  Residual(MolSys& m_, BulkSys& bs_) : m(m_), bs(bs_) {
    const auto inr = species_in_reactions(m);
    for (size_t i = 0; i < m.species.size(); i++) {
      if (!std::isnan(m.pS[i])) ph_species.push_back((int)i);
      else if (inr.count(m.species[i])) rxn_species.push_back((int)i);
    }
    n = rxn_species.size() + ph_species.size() + 1;
  }
  std::vector<double> initial(const Bulk& b) const {
    std::vector<double> x;
    for (int i : rxn_species) x.push_back(std::log(b.rho_species[i]));
    for (int i : ph_species) x.push_back(std::log(b.rho_species[i]));
    x.push_back(0.0);
    return x;
  }
  // residual_bulkstate.jl:26-35 with update_bulk_structures.jl:10-44 and eval_residuals.jl:26-60
  std::vector<double> operator()(Bulk& b, const std::vector<double>& x, std::vector<char>& adjustable) const {
    balance_charge(m, b, x.back(), adjustable);
    const auto inr = species_in_reactions(m);
    size_t ir = 0, ip = 0;
    for (size_t i = 0; i < m.species.size(); i++) {
      if (!std::isnan(m.pS[i])) b.rho_species[i] = std::exp(x[rxn_species.size() + ip++]);
      else if (inr.count(m.species[i])) b.rho_species[i] = std::exp(x[ir++]);
    }
    std::vector<double> lng_in(b.lng);
    lng_in.push_back(0.0);
    b.segs.assign(bs.seg_total + 1, 0.0);
    std::vector<double> rbo(b.rho_bonds.size() + 1, 0.0), mu(b.mu_ex.size()), lng(b.lng.size() + 1), mus(b.mu_species.size());
    std::vector<double> xi(b.Xi.size());
    const int rc = sdft_bulk_eval(&bs.sys, b.rho_species.data(), b.mu_ex.data(), lng_in.data(), b.segs.data(),
                                  b.rho_beads.data(), rbo.data(), mus.data(), mu.data(), lng.data(), xi.data());
    if (rc != SDFT_OK) fail("bulk evaluation failed");
    std::copy(rbo.begin(), rbo.begin() + b.rho_bonds.size(), b.rho_bonds.begin());
    b.mu_species = mus;
    b.mu_ex = mu;
    std::copy(lng.begin(), lng.begin() + b.lng.size(), b.lng.begin());
    b.Xi = xi;
    std::vector<double> res;
    const double unit = concentration_to_density(1.0, m.c);
    for (size_t i = 0; i < m.species.size(); i++)
      if (!std::isnan(m.pS[i])) res.push_back(b.mu_species[i] + m.pS[i] * kLog10 - std::log(unit));
    for (const auto& r : m.reactions) {
      if (r.bookkeeping()) continue;
      double musum = 0.0;
      for (size_t k = 0; k < r.species.size(); k++) {
        auto it = std::find(m.species.begin(), m.species.end(), r.species[k]);
        if (it == m.species.end()) fail("reaction species " + r.species[k] + " is not a species");
        musum += r.coeffs[k] * b.mu_species[it - m.species.begin()];
      }
      res.push_back(musum - r.pK);
    }
    std::vector<double> qr(m.species.size());
    for (size_t i = 0; i < qr.size(); i++) qr[i] = m.charge[i] * b.rho_species[i];
    res.push_back(-np_sum(qr.data(), qr.size()));
    // the driver subtracts the residual from the unknowns (AndersonResidual.jl:27-138)
    if (res.size() != n)
      fail("bulk state: " + std::to_string(res.size()) + " equations for " + std::to_string(n) + " unknowns");
    return res;
  }
};

double max_abs(const std::vector<double>& v) {
  double m = 0.0;
  for (double a : v) m = std::max(m, std::fabs(a));
  return m;
}
bool all_finite(const std::vector<double>& v) {
  for (double a : v)
    if (!std::isfinite(a)) return false;
  return true;
}
double dot(const double* a, const double* b, size_t n) {
  double s = 0.0;
  for (size_t i = 0; i < n; i++) s += a[i] * b[i];
  return s;
}
double nrm2(const std::vector<double>& v) { return std::sqrt(dot(v.data(), v.data(), v.size())); }

// LSQR (Paige & Saunders, ACM TOMS 8(1):43-71, 1982) with IterativeSolvers.jl's
// defaults: atol = btol = sqrt(eps), conlim = 1/sqrt(eps), maxiter = max(m, n), no
// damping, x the warm start.  A is m x k, column-major.
void lsqr(std::vector<double>& x, const std::vector<double>& A, size_t m, size_t k, const std::vector<double>& b) {
  const double eps = DBL_EPSILON, atol = std::sqrt(eps), btol = std::sqrt(eps), ctol = std::sqrt(eps);
  const size_t maxiter = std::max(m, k);
  auto Av = [&](const std::vector<double>& v) {
    std::vector<double> o(m, 0.0);
    for (size_t j = 0; j < k; j++)
      for (size_t i = 0; i < m; i++) o[i] += A[j * m + i] * v[j];
    return o;
  };
  auto ATu = [&](const std::vector<double>& u) {
    std::vector<double> o(k);
    for (size_t j = 0; j < k; j++) o[j] = dot(&A[j * m], u.data(), m);
    return o;
  };
  std::vector<double> u = Av(x);
  for (size_t i = 0; i < m; i++) u[i] = b[i] - u[i];
  std::vector<double> v(k, 0.0);
  double alpha = 0.0, beta = nrm2(u);
  if (beta > 0) {
    for (double& a : u) a /= beta;
    v = ATu(u);
    alpha = nrm2(v);
  }
  if (alpha > 0)
    for (double& a : v) a /= alpha;
  std::vector<double> w = v;
  double arnorm = alpha * beta;
  if (arnorm == 0) return;
  double anorm = 0, acond = 0, ddnorm = 0, res2 = 0, xxnorm = 0, z = 0, sn2 = 0, cs2 = -1.0;
  double rhobar = alpha, phibar = beta, bnorm = beta;
  size_t itn = 0;
  int istop = 0;
  while (itn < maxiter && istop == 0) {
    itn++;
    std::vector<double> Avv = Av(v);
    for (size_t i = 0; i < m; i++) u[i] = Avv[i] - alpha * u[i];
    beta = nrm2(u);
    if (beta > 0) {
      for (double& a : u) a /= beta;
      anorm = std::sqrt(anorm * anorm + alpha * alpha + beta * beta);
      std::vector<double> t = ATu(u);
      for (size_t j = 0; j < k; j++) v[j] = t[j] - beta * v[j];
      alpha = nrm2(v);
      if (alpha > 0)
        for (double& a : v) a /= alpha;
    }
    const double rho = std::sqrt(rhobar * rhobar + beta * beta);
    const double cs = rhobar / rho, sn = beta / rho, theta = sn * alpha;
    rhobar = -cs * alpha;
    const double phi = cs * phibar;
    phibar = sn * phibar;
    const double tau = sn * phi, t1 = phi / rho, t2 = -theta / rho;
    double dkk = 0.0;
    for (size_t j = 0; j < k; j++) {
      const double dk = w[j] / rho;
      dkk += dk * dk;
      x[j] += t1 * w[j];
      w[j] = v[j] + t2 * w[j];
    }
    ddnorm += dkk;
    const double delta = sn2 * rho, gambar = -cs2 * rho, rhs = phi - delta * z, zbar = rhs / gambar;
    const double xnorm = std::sqrt(xxnorm + zbar * zbar), gamma = std::sqrt(gambar * gambar + theta * theta);
    cs2 = gambar / gamma;
    sn2 = theta / gamma;
    z = rhs / gamma;
    xxnorm += z * z;
    acond = anorm * std::sqrt(ddnorm);
    const double res1 = phibar * phibar, rnorm = std::sqrt(res1 + res2);
    arnorm = alpha * std::fabs(tau);
    const double test1 = rnorm / bnorm, test2 = arnorm / (anorm * rnorm), test3 = 1.0 / acond;
    const double t1b = test1 / (1.0 + anorm * xnorm / bnorm), rtol = btol + atol * anorm * xnorm / bnorm;
    if (itn >= maxiter) istop = 7;
    if (1.0 + test3 <= 1.0) istop = 6;
    if (1.0 + test2 <= 1.0) istop = 5;
    if (1.0 + t1b <= 1.0) istop = 4;
    if (test3 <= ctol) istop = 3;
    if (test2 <= atol) istop = 2;
    if (test1 <= rtol) istop = 1;
  }
}

// min-norm least squares of an m x k column-major matrix (k small) by one-sided
// Jacobi SVD, singular values below eps * max(m, k) * s_max dropped (numpy's
// lstsq with rcond=None)
std::vector<double> lstsq(std::vector<double> A, size_t m, size_t k, const std::vector<double>& b) {
  std::vector<double> V(k * k, 0.0);
  for (size_t j = 0; j < k; j++) V[j * k + j] = 1.0;
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0.0;
    for (size_t p = 0; p < k; p++)
      for (size_t q = p + 1; q < k; q++) {
        double* ap = &A[p * m];
        double* aq = &A[q * m];
        const double alpha = dot(ap, ap, m), beta = dot(aq, aq, m), gamma = dot(ap, aq, m);
        if (gamma == 0.0) continue;
        off = std::max(off, std::fabs(gamma) / std::sqrt(alpha * beta));
        const double zeta = (beta - alpha) / (2.0 * gamma);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
        const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
        for (size_t i = 0; i < m; i++) {
          const double x = ap[i], y = aq[i];
          ap[i] = c * x - s * y;
          aq[i] = s * x + c * y;
        }
        for (size_t i = 0; i < k; i++) {
          const double x = V[p * k + i], y = V[q * k + i];
          V[p * k + i] = c * x - s * y;
          V[q * k + i] = s * x + c * y;
        }
      }
    if (off < 1e-15) break;
  }
  std::vector<double> sv(k);
  double smax = 0.0;
  for (size_t j = 0; j < k; j++) smax = std::max(smax, sv[j] = std::sqrt(dot(&A[j * m], &A[j * m], m)));
  const double cut = DBL_EPSILON * (double)std::max(m, k) * smax;
  std::vector<double> x(k, 0.0);
  for (size_t j = 0; j < k; j++) {
    if (!(sv[j] > cut)) continue;
    const double c = dot(&A[j * m], b.data(), m) / (sv[j] * sv[j]);  // (u_j . b) / s_j with u_j = a_j / s_j
    for (size_t i = 0; i < k; i++) x[i] += V[j * k + i] * c;
  }
  return x;
}

struct BulkDiverged {};

std::map<std::string, double> bulk_numerics(const Node* numerical) {
  std::map<std::string, double> num{{"mixing_max", 0.1}, {"tole", 1e-10}, {"damping", 0.1}};
  if (numerical && numerical->kind == Node::Map)
    for (const auto& kv : numerical->map) num[kv.first] = as_float(kv.second);
  return num;
}
double numv(const std::map<std::string, double>& n, const char* k, double d) {
  auto it = n.find(k);
  return it == n.end() ? d : it->second;
}

// Int(x) of AndersonMixing.jl:74-79: a finite integral value, or an error.
// max_iters beyond the int32 range of sdft_numerics is clamped (a count that
// large is never reached); anderm must fit.
int32_t numerics_int(const std::map<std::string, double>& n, const char* key, int32_t def, bool clamp) {
  const double v = numv(n, key, def);
  if (!std::isfinite(v) || v != std::floor(v) || (!clamp && (v < INT32_MIN || v > INT32_MAX)))
    fail(std::string("numerical.") + key + " must be an integer");
  return (int32_t)std::max<double>(INT32_MIN, std::min<double>(INT32_MAX, v));
}

// AndersonResidual.jl:27-138 (restated driver)
Bulk solve_bulk_reference(MolSys& m, BulkSys& bs, const std::map<std::string, double>& num, int cap) {
  Bulk b = initialize_densities(m);
  const long max_iters = numerics_int(num, "max_iters", 100000, true);
  const double damping = numv(num, "damping", 0.1), mix_max = numv(num, "mixing_max", 0.1);
  const double switch_mix = numv(num, "switch_mix", 1e-4), tole = numv(num, "tole", 1e-6);
  const int mm = numerics_int(num, "anderm", 5, false);
  std::vector<char> adjustable(m.adjustable);
  Residual R(m, bs);
  std::vector<double> Xk = R.initial(b);
  const size_t n = Xk.size();
  std::vector<double> X(n * mm, 0.0), F(n * mm, 0.0);
  std::vector<double> Fk = R(b, Xk, adjustable);
  for (size_t i = 0; i < n; i++) X[i] = Xk[i], F[i] = Fk[i];
  std::vector<double> lambdas(mm - 1, 0.0);
  long it = 0;
  double err = 1.0;
  while (it < max_iters) {
    it++;
    if (it > cap) throw BulkDiverged{};
    Fk = R(b, Xk, adjustable);
    if (!all_finite(Fk)) throw BulkDiverged{};
    err = std::max(max_abs(Fk), 1e-20);
    const double amix = std::min(mix_max, damping / err);
    const int col = (int)(it % mm);
    for (size_t i = 0; i < n; i++) X[col * n + i] = Xk[i], F[col * n + i] = Fk[i];
    if (it < mm || err > switch_mix) {
      const int prev = (int)((it - 1) % mm);
      std::vector<double> dX(n), dF(n);
      for (size_t i = 0; i < n; i++) dX[i] = Xk[i] - X[prev * n + i], dF[i] = Fk[i] - F[prev * n + i];
      const double numer = dot(Fk.data(), dF.data(), n), denom = dot(dF.data(), dF.data(), n);
      const double lam = denom == 0.0 ? 0.0 : numer / denom;
      for (size_t i = 0; i < n; i++) Xk[i] = Xk[i] - lam * dX[i] - amix * (Fk[i] - lam * dF[i]);
    } else {
      std::vector<double> tX, tF, negF(n);
      for (int j = 0; j < mm; j++) {
        if (j == col) continue;
        for (size_t i = 0; i < n; i++) tX.push_back(X[j * n + i] - Xk[i]), tF.push_back(F[j * n + i] - Fk[i]);
      }
      for (size_t i = 0; i < n; i++) negF[i] = -Fk[i];
      lsqr(lambdas, tF, n, mm - 1, negF);
      for (size_t i = 0; i < n; i++) {
        double a = 0.0, c = 0.0;
        for (int j = 0; j < mm - 1; j++) a += tX[j * n + i] * lambdas[j], c += tF[j * n + i] * lambdas[j];
        Xk[i] = Xk[i] + a + amix * (Fk[i] + c);
      }
    }
    if (err < tole) break;
  }
  b.iterations = (int)it;
  b.residual = err;
  return b;
}

// undamped Picard x <- x - F(x) with Anderson mixing (type II, depth 5)
Bulk solve_bulk_robust(MolSys& m, BulkSys& bs, const std::map<std::string, double>& num) {
  const double tole = std::min(numv(num, "tole", 1e-6), 1e-10);
  Bulk b = initialize_densities(m);
  std::vector<char> adjustable(m.adjustable);
  Residual R(m, bs);
  std::vector<double> Xk = R.initial(b);
  const size_t n = Xk.size();
  const int depth = 5;
  std::vector<std::vector<double>> hx, hf;
  double err = INFINITY;
  int it = 1;
  for (; it <= 2000; it++) {
    std::vector<double> Fk = R(b, Xk, adjustable);
    if (!all_finite(Fk)) fail("bulk solve: non-finite residual");
    err = max_abs(Fk);
    if (err < tole) break;
    std::vector<double> G(n);
    for (size_t i = 0; i < n; i++) G[i] = Xk[i] - Fk[i];
    hx.push_back(Xk);
    hf.push_back(Fk);
    if ((int)hx.size() > depth) {
      hx.erase(hx.begin());
      hf.erase(hf.begin());
    }
    if (hx.size() >= 2) {
      const size_t k = hx.size() - 1;
      std::vector<double> dF(n * k), dXmF(n * k);
      for (size_t j = 0; j < k; j++)
        for (size_t i = 0; i < n; i++) {
          dF[j * n + i] = hf[j + 1][i] - hf[j][i];
          dXmF[j * n + i] = (hx[j + 1][i] - hx[j][i]) - dF[j * n + i];
        }
      const std::vector<double> gam = lstsq(dF, n, k, Fk);
      for (size_t i = 0; i < n; i++) {
        double s = 0.0;
        for (size_t j = 0; j < k; j++) s += dXmF[j * n + i] * gam[j];
        Xk[i] = G[i] - s;
      }
    } else {
      Xk = G;
    }
  }
  if (it > 2000) fail("bulk solve did not converge");
  b.iterations = it;
  b.residual = err;
  return b;
}

// solver_bulkstate.jl:31-62: the restated driver first; if it diverges, the robust form
Bulk solve_bulk(MolSys& m, const Node* numerical) {
  BulkSys bs;
  build_bulk_sys(m, bs);
  const auto num = bulk_numerics(numerical);
  const std::vector<double> charge0 = m.charge;
  // zeros(n, anderm) of the history (AndersonResidual.jl) needs anderm >= 1
  if (numerics_int(num, "anderm", 5, false) < 1) fail("numerical.anderm must be at least 1");
  numerics_int(num, "max_iters", 100000, true);
  try {
    return solve_bulk_reference(m, bs, num, 3000);
  } catch (const BulkDiverged&) {
  } catch (const InputError& e) {
    if (std::string(e.what()).find("No compensating species") != std::string::npos) throw;
  }
  m.charge = charge0;
  return solve_bulk_robust(m, bs, num);
}

}  // namespace

int sdft_record_error(int code, const std::string& msg);  // softdft.cu: the text of sdft_last_error

namespace {

// ===========================================================================
// geometry and descriptor
// ===========================================================================
// Julia's cld on Float64: the ceiling of the exact quotient x / y (y > 0)
long cld_exact(double x, double y) {
  if (!(y > 0) || !std::isfinite(x) || !std::isfinite(y)) fail("bin_width must be positive and finite");
  if (!(x >= 0) || x / y > 1e8) fail("the slit needs 0 <= dimensions / bin_width <= 1e8");
  long k = (long)std::ceil(x / y);
  while (std::fma((double)k, y, -x) < 0) k++;        // k y < x
  while (std::fma((double)(k - 1), y, -x) >= 0) k--;  // (k - 1) y >= x
  return k;
}
long julia_round(double x) { return (long)std::nearbyint(x); }  // round half to even

struct Slit {
  double H = 0, dz = 0;
  long NP = 0;
  bool hard = false, charged = false;
  double q[2] = {0, 0};
};

// create_cartesian.jl:66 (NP = cld(H, dz) + 1), external_fields.jl:11-24
Slit geometry_system(const Node& ds) {
  const Node* g = ds.get("geometry");
  if (!g) fail("Missing required section: 'geometry'.");
  const Node* cs = g->get("coordinate_system");
  if (!cs) fail("Missing required key: 'coordinate_system' under 'geometry'.");
  if (as_str(*cs) != "Cartesian") fail("Unknown coordinate system: " + as_str(*cs) + ". Supported: Cartesian.");
  const Node* dims = g->get("dimensions");
  const Node* bins = g->get("bin_width");
  if (!dims || !bins) fail("Please specify both `dimensions` and `bin_width` under `geometry`.");
  if (dims->kind != Node::Seq || bins->kind != Node::Seq || dims->seq.size() != bins->seq.size())
    fail("Mismatch in number of `dimensions` and `bin_width` entries.");
  if (dims->seq.size() != 1) fail("only the 1D Cartesian slit is supported by the device solve", SDFT_ERR_UNSUPPORTED);
  Slit s;
  s.H = as_float(dims->seq[0]);
  s.dz = as_float(bins->seq[0]);
  s.NP = cld_exact(s.H, s.dz) + 1;
  const Node* ext = g->get("external_field");
  if (ext && ext->kind == Node::Map)
    for (const auto& kv : ext->map) {
      const Node& d = kv.second;
      if (kv.first == "hard_walls") {
        const Node* dd = d.get("dims");
        if (!dd || dd->kind == Node::Null) fail("Missing 'dims' key in external_field[:hard_walls].");
        for (const Node& x : listed(*dd)) {
          if (as_int(x) != 1) fail("Invalid dimension index: " + as_str(x));
          s.hard = true;
        }
      } else if (kv.first == "charged_walls") {
        const Node* dp = d.get("dims");
        if (!dp || dp->kind == Node::Null) fail("Please specify the dimensions using 'dims: [i, j, ...]'.");
        const std::vector<Node> dd = listed(*dp);
        const Node* ch = d.get("charge");
        if (!ch) fail("Please specify wall charges under 'charge'.");
        std::vector<const Node*> rows;
        if (!ch->seq.empty() && ch->seq[0].kind != Node::Seq) rows.push_back(ch);
        else
          for (const Node& r : ch->seq) rows.push_back(&r);
        if (rows.size() != dd.size()) fail("Mismatch: number of charge entries does not match dims.");
        for (size_t i = 0; i < dd.size(); i++) {
          if (as_int(dd[i]) != 1) fail("Invalid dimension index in dims");
          if (rows[i]->seq.size() < 2) fail("wall charges need two values");
          s.charged = true;
          s.q[0] = as_float(rows[i]->seq[0]);
          s.q[1] = as_float(rows[i]->seq[1]);
        }
      } else {
        fail("external field '" + kv.first + "' is not supported by the device solve", SDFT_ERR_UNSUPPORTED);
      }
    }
  return s;
}

}  // namespace

// a parsed input.yaml: the descriptor of sdft_request_create and the arrays it points into
struct sdft_input {
  sdft_system_desc desc{};
  std::vector<sdft_species_desc> sp;
  std::vector<std::vector<int32_t>> ints;
  std::vector<std::vector<double>> dbls;
  sdft_numerics num{};
  int bulk_iterations = 0;
  double bulk_residual = 0.0;
  const int32_t* keep(std::vector<int32_t> v) {
    if (v.empty()) v.push_back(0);
    ints.push_back(std::move(v));
    return ints.back().data();
  }
  const double* keep(std::vector<double> v) {
    if (v.empty()) v.push_back(0.0);
    dbls.push_back(std::move(v));
    return dbls.back().data();
  }
};

namespace {

// fixed (grafted) segments: determine_fixed.jl:1-29 (wall index +- round(sigma / 2 dz))
void fixed_segments(const Node& ds, const MolSys& m, const Slit& g, size_t u, std::vector<int32_t>& coords,
                    double* dens) {
  const Config& cfg = m.configs[u];
  coords.assign(cfg.sequence.size(), -1);
  *dens = 0.0;
  const Node& entry = ds.get("species")->seq[u];
  const Node* fx = entry.get("fixed");
  if (!fx) return;
  if (m.densities[u] > 0.0)
    fail("Species " + std::to_string(u + 1) +
         " defines a fixed segment but also has nonzero input density. Simultaneous bulk and brush densities are not supported.");
  if (!fx->has("density")) fail("Species " + std::to_string(u + 1) + " contains 'fixed' but does not specify a density.");
  *dens = as_float(*fx->get("density"));
  const Node* segs = fx->get("segment");
  const Node* pos = fx->get("position");
  if (!segs || !pos) fail("Species " + std::to_string(u + 1) + " contains 'fixed' but is missing 'segment' or 'position'.");
  if (segs->seq.size() != pos->seq.size())
    fail("Mismatch in number of fixed segments and specified positions for species " + std::to_string(u + 1) + ".");
  const long idx_LW = julia_round(0.0 / g.dz) + 1, idx_RW = julia_round(g.H / g.dz) + 1;
  for (size_t k = 0; k < segs->seq.size(); k++) {
    const int L = as_int(segs->seq[k]);
    if (L < 1 || L > (int)cfg.sequence.size()) fail("fixed segment index out of range");
    const int j = cfg.sequence[L - 1];
    const long dzr = julia_round(m.diameters[j] / g.dz / 2.0);
    const std::string tag = as_str(pos->seq[k]);
    long c1;
    if (tag == "left") c1 = idx_LW + dzr;
    else if (tag == "right") c1 = idx_RW - dzr;
    else fail("Invalid grafting position tag for species " + std::to_string(u + 1) + ": '" + tag + "'");
    coords[L - 1] = (int32_t)(c1 - 1);
  }
  for (size_t g2 = 1; g2 < coords.size(); g2++)
    if (coords[g2] >= 0)
      fail("Species " + std::to_string(u + 1) + ": only the first segment can be fixed in a 1D slit", SDFT_ERR_UNSUPPORTED);
}

// AndersonMixing.jl:74-79 defaults over the numerical section
sdft_numerics numerics_of(const Node& ds) {
  std::map<std::string, double> n;
  if (const Node* num = ds.get("numerical"))
    if (num->kind == Node::Map)
      for (const auto& kv : num->map) n[kv.first] = as_float(kv.second);
  sdft_numerics o;
  o.max_iters = numerics_int(n, "max_iters", 100000, true);
  o.anderm = numerics_int(n, "anderm", 5, false);
  o.damping = numv(n, "damping", 0.5);
  o.mixing_max = numv(n, "mixing_max", 1.0);
  o.switch_tole = numv(n, "switch_tole", 1e-3);
  o.tole = numv(n, "tole", 1e-6);
  o.mixed_switch = numv(n, "mixed_switch", 0.0);
  return o;
}

void build(const std::string& text, sdft_input& in) {
  const Node ds = load_yaml(text);
  MolSys m = molecular_system(ds);
  const Bulk b = solve_bulk(m, ds.get("numerical"));
  const Slit g = geometry_system(ds);
  uint32_t funcs = 0;
  for (const auto& f : m.fe_model) {
    if (f == "mfmt") funcs |= SDFT_FUNC_MFMT;
    else if (f == "TPT1mfmt") funcs |= SDFT_FUNC_TPT1MFMT;
    else if (f == "msa") funcs |= SDFT_FUNC_MSA;
    else if (f == "TPT1msa") funcs |= SDFT_FUNC_TPT1MSA;
    else if (f != "ideal" && f != "coul") fail("functional '" + f + "' is not supported by the device solve", SDFT_ERR_UNSUPPORTED);
  }
  const size_t ns = m.configs.size();
  in.ints.reserve(6 * ns + 4);
  in.dbls.reserve(ns + 8);
  in.sp.resize(ns);
  for (size_t u = 0; u < ns; u++) {
    const Config& cfg = m.configs[u];
    if (cfg.model != "freely_jointed") fail("monomerbead species are not supported by the device solve", SDFT_ERR_UNSUPPORTED);
    const int n = (int)cfg.sequence.size();
    int S = 1;
    for (const auto& f : cfg.family) S = std::max(S, (int)f.size());
    std::vector<int32_t> parent, nst, st((size_t)n * S, -1), coords;
    for (int gg = 0; gg < n; gg++) {
      if (cfg.topo.parents[gg].size() > 1) fail("segments with more than one parent are not supported", SDFT_ERR_UNSUPPORTED);
      parent.push_back(cfg.topo.parents[gg].empty() ? -1 : cfg.topo.parents[gg][0]);
      nst.push_back((int)cfg.family[gg].size());
      for (size_t i = 0; i < cfg.family[gg].size(); i++) st[(size_t)gg * S + i] = cfg.family[gg][i];
    }
    double dens;
    fixed_segments(ds, m, g, u, coords, &dens);
    bool any_fixed = false;
    for (int32_t c : coords) any_fixed |= c >= 0;
    sdft_species_desc& s = in.sp[u];
    s.n_seg = n;
    s.max_states = S;
    s.parent = in.keep(parent);
    s.n_states = in.keep(nst);
    s.states = in.keep(st);
    s.fixed_coord = in.keep(coords);
    s.fixed_density = dens;
    if (any_fixed && n > 20000)
      fail("grafted chains of more than 20000 segments are not supported (path-length matrix of n^2 entries)",
           SDFT_ERR_UNSUPPORTED);
    s.max_distance = any_fixed ? in.keep(max_distance_matrix(cfg, m.diameters)) : nullptr;
    s.mu_species = b.mu_species[u];
  }
  std::vector<int32_t> bonds;
  for (const auto& bd : m.bonds) {
    bonds.push_back(bd.first);
    bonds.push_back(bd.second);
  }
  sdft_system_desc& d = in.desc;
  d.abi_version = SDFT_ABI_VERSION;
  d.np = (int32_t)g.NP;
  d.bin_width = g.dz;
  d.length = g.H;
  d.hard_walls = g.hard ? 1 : 0;
  d.charged_walls = g.charged ? 1 : 0;
  d.wall_charge[0] = g.q[0];
  d.wall_charge[1] = g.q[1];
  d.bjerrum_length = m.bjerrum;
  d.nb = (int32_t)m.monomers.size();
  d.diameter = in.keep(m.diameters);
  d.valence = in.keep(m.valences);
  d.delta_muH = in.keep(m.dmu);
  d.mb = (int32_t)m.bonds.size();
  d.bond_types = in.keep(bonds);
  d.n_species = (int32_t)ns;
  d.species = in.sp.data();
  d.functionals = funcs;
  d.mu_ex_bulk = in.keep(b.mu_ex);
  d.lng_bulk = in.keep(b.lng);
  in.num = numerics_of(ds);
  in.bulk_iterations = b.iterations;
  in.bulk_residual = b.residual;
}

}  // namespace

extern "C" int sdft_input_from_yaml(const char* yaml_text, sdft_input** out) {
  if (!yaml_text || !out) return sdft_record_error(SDFT_ERR_ARG, "null argument");
  *out = nullptr;
  auto in = std::make_unique<sdft_input>();
  try {
    build(yaml_text, *in);
  } catch (const InputError& e) {
    return sdft_record_error(e.code, e.what());
  } catch (const std::exception& e) {
    return sdft_record_error(SDFT_ERR_ARG, e.what());
  }
  *out = in.release();
  return SDFT_OK;
}

extern "C" const sdft_system_desc* sdft_input_descriptor(const sdft_input* in) { return in ? &in->desc : nullptr; }

extern "C" int sdft_input_numerics(const sdft_input* in, sdft_numerics* out) {
  if (!in || !out) return sdft_record_error(SDFT_ERR_ARG, "null argument");
  *out = in->num;
  return SDFT_OK;
}

extern "C" int sdft_input_bulk_stats(const sdft_input* in, int32_t* iterations, double* residual) {
  if (!in) return sdft_record_error(SDFT_ERR_ARG, "null argument");
  if (iterations) *iterations = in->bulk_iterations;
  if (residual) *residual = in->bulk_residual;
  return SDFT_OK;
}

extern "C" int sdft_input_destroy(sdft_input* in) {
  delete in;
  return SDFT_OK;
}
