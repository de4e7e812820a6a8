// urdf.cpp -- native URDF / model-directive loader producing the flat
// MinimalPlant tables of csd_plant_desc_t, for callers without Python.
//
// Reference: URDFParser (csdecomp/src/plant/urdf_parser.cpp:78-206 parse and
// finalize, :208-466 joints/links/geometries, :485-616 scene grouping and
// collision-pair filter, :618-778 directives) over tinyxml2 and yaml-cpp, and
// KinematicTree::finalize (kinematic_tree.cpp:82-146). Neither library is
// available here, so this file carries its own small XML reader (elements
// and attributes; comments, declarations and text skipped) and a reader for
// the YAML subset model directives use (block mappings and sequences, flow
// sequences and mappings, tags ignored, comments). The URDF rules are the
// ones csdecomp_b200/plant.py states (links before joints, rpy = Rz Ry Rx in
// double rounded to float, box sizes are full extents, sphere dimensions
// (r, -1, -1), capsules (r, length, r)); numbers are read as double and
// rounded to float, as the Python loader reads them.
#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <sys/stat.h>
#include <unordered_map>
#include <vector>

#include "../../include/csd_capi.h"

namespace csd {

void set_error(const std::string& msg);  // capi error slot of the calling thread

#define CSD_CHECK(cond, code, msg) \
  do {                             \
    if (!(cond)) {                 \
      ::csd::set_error(msg);       \
      return (code);               \
    }                              \
  } while (0)

namespace urdf {

// ------------------------------------------------------------------ XML
struct XmlNode {
  std::string tag;
  std::vector<std::pair<std::string, std::string>> attrs;
  std::vector<XmlNode> children;

  const std::string* attr(const char* name) const {
    for (const auto& a : attrs)
      if (a.first == name) return &a.second;
    return nullptr;
  }
  void set_attr(const char* name, const std::string& v) {
    for (auto& a : attrs)
      if (a.first == name) {
        a.second = v;
        return;
      }
    attrs.emplace_back(name, v);
  }
  const XmlNode* child(const char* tag_name) const {
    for (const auto& c : children)
      if (c.tag == tag_name) return &c;
    return nullptr;
  }
};

class XmlReader {
 public:
  explicit XmlReader(const std::string& s) : s_(s) {}

  XmlNode parse_document() {
    skip_misc();
    if (i_ >= s_.size() || s_[i_] != '<') fail("no root element");
    XmlNode root = parse_element();
    skip_misc();
    if (i_ != s_.size()) fail("content after the root element");
    return root;
  }

 private:
  const std::string& s_;
  size_t i_ = 0;

  [[noreturn]] void fail(const std::string& what) const {
    throw std::runtime_error("XML parse error at offset " + std::to_string(i_) + ": " + what);
  }
  bool starts(const char* p) const { return s_.compare(i_, std::strlen(p), p) == 0; }
  void skip_ws() {
    while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
  }
  void skip_until(const char* end) {
    const size_t e = s_.find(end, i_);
    if (e == std::string::npos) fail(std::string("unterminated construct, expected ") + end);
    i_ = e + std::strlen(end);
  }
  // whitespace, comments, declarations and processing instructions
  void skip_misc() {
    for (;;) {
      skip_ws();
      if (starts("<!--")) {
        skip_until("-->");
      } else if (starts("<?")) {
        skip_until("?>");
      } else if (starts("<!")) {
        // DOCTYPE, with an optional internal subset in brackets
        int depth = 0;
        for (; i_ < s_.size(); ++i_) {
          if (s_[i_] == '[') ++depth;
          if (s_[i_] == ']') --depth;
          if (s_[i_] == '>' && depth <= 0) break;
        }
        if (i_ >= s_.size()) fail("unterminated declaration");
        ++i_;
      } else {
        return;
      }
    }
  }
  std::string parse_name() {
    const size_t b = i_;
    while (i_ < s_.size()) {
      const char c = s_[i_];
      if (std::isspace((unsigned char)c) || c == '=' || c == '>' || c == '/' || c == '<') break;
      ++i_;
    }
    if (i_ == b) fail("expected a name");
    return s_.substr(b, i_ - b);
  }
  static void append_utf8(std::string* out, unsigned long cp) {
    if (cp < 0x80) {
      out->push_back((char)cp);
    } else if (cp < 0x800) {
      out->push_back((char)(0xC0 | (cp >> 6)));
      out->push_back((char)(0x80 | (cp & 0x3F)));
    } else if (cp < 0x10000) {
      out->push_back((char)(0xE0 | (cp >> 12)));
      out->push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      out->push_back((char)(0x80 | (cp & 0x3F)));
    } else {
      out->push_back((char)(0xF0 | (cp >> 18)));
      out->push_back((char)(0x80 | ((cp >> 12) & 0x3F)));
      out->push_back((char)(0x80 | ((cp >> 6) & 0x3F)));
      out->push_back((char)(0x80 | (cp & 0x3F)));
    }
  }
  std::string decode(const std::string& raw) const {
    std::string out;
    for (size_t k = 0; k < raw.size(); ++k) {
      if (raw[k] != '&') {
        out.push_back(raw[k]);
        continue;
      }
      const size_t e = raw.find(';', k);
      if (e == std::string::npos) fail("unterminated entity");
      const std::string ent = raw.substr(k + 1, e - k - 1);
      if (ent == "lt") out.push_back('<');
      else if (ent == "gt") out.push_back('>');
      else if (ent == "amp") out.push_back('&');
      else if (ent == "quot") out.push_back('"');
      else if (ent == "apos") out.push_back('\'');
      else if (ent.size() > 1 && ent[0] == '#')
        append_utf8(&out, ent[1] == 'x' ? std::strtoul(ent.c_str() + 2, nullptr, 16)
                                        : std::strtoul(ent.c_str() + 1, nullptr, 10));
      else fail("unknown entity &" + ent + ";");
      k = e;
    }
    return out;
  }
  XmlNode parse_element() {
    ++i_;  // '<'
    XmlNode n;
    n.tag = parse_name();
    for (;;) {
      skip_ws();
      if (i_ >= s_.size()) fail("unterminated start tag");
      if (starts("/>")) {
        i_ += 2;
        return n;
      }
      if (s_[i_] == '>') {
        ++i_;
        break;
      }
      std::string an = parse_name();
      skip_ws();
      if (i_ >= s_.size() || s_[i_] != '=') fail("expected '=' after attribute " + an);
      ++i_;
      skip_ws();
      if (i_ >= s_.size() || (s_[i_] != '"' && s_[i_] != '\'')) fail("expected a quoted attribute value");
      const char q = s_[i_++];
      const size_t e = s_.find(q, i_);
      if (e == std::string::npos) fail("unterminated attribute value");
      n.attrs.emplace_back(an, decode(s_.substr(i_, e - i_)));
      i_ = e + 1;
    }
    // content: child elements; text, comments, CDATA and instructions skipped
    for (;;) {
      const size_t lt = s_.find('<', i_);
      if (lt == std::string::npos) fail("unterminated element " + n.tag);
      i_ = lt;
      if (starts("</")) {
        i_ += 2;
        const std::string close = parse_name();
        if (close != n.tag) fail("mismatched end tag </" + close + "> for <" + n.tag + ">");
        skip_ws();
        if (i_ >= s_.size() || s_[i_] != '>') fail("malformed end tag");
        ++i_;
        return n;
      }
      if (starts("<!--")) {
        skip_until("-->");
      } else if (starts("<![CDATA[")) {
        skip_until("]]>");
      } else if (starts("<?")) {
        skip_until("?>");
      } else {
        n.children.push_back(parse_element());
      }
    }
  }
};

// ------------------------------------------------------------------ YAML subset
struct YNode {
  enum Kind { SCALAR, SEQ, MAP } kind = SCALAR;
  std::string scalar;
  std::vector<YNode> seq;
  std::vector<std::pair<std::string, YNode>> map;

  const YNode* get(const char* key) const {
    for (const auto& kv : map)
      if (kv.first == key) return &kv.second;
    return nullptr;
  }
};

class YamlReader {
 public:
  explicit YamlReader(const std::string& text) {
    std::istringstream in(text);
    std::string line;
    int no = 0;
    while (std::getline(in, line)) {
      ++no;
      const std::string body = strip_comment(line);
      size_t ind = 0;
      while (ind < body.size() && body[ind] == ' ') ++ind;
      if (ind == body.size()) continue;
      if (body[ind] == '\t') throw std::runtime_error("YAML: tab indentation on line " + std::to_string(no));
      std::string rest = body.substr(ind);
      while (!rest.empty() && std::isspace((unsigned char)rest.back())) rest.pop_back();
      if (rest == "---" || rest == "...") continue;
      lines_.push_back({(int)ind, rest, no});
    }
  }

  YNode parse() {
    size_t k = 0;
    if (lines_.empty()) return YNode{};
    YNode n = parse_block(k, lines_[0].indent);
    if (k != lines_.size()) throw std::runtime_error("YAML: unexpected content on line " + std::to_string(lines_[k].no));
    return n;
  }

 private:
  struct Line {
    int indent;
    std::string text;
    int no;
  };
  std::vector<Line> lines_;

  static std::string strip_comment(const std::string& s) {
    bool sq = false, dq = false;
    for (size_t k = 0; k < s.size(); ++k) {
      const char c = s[k];
      if (c == '\'' && !dq) sq = !sq;
      else if (c == '"' && !sq) dq = !dq;
      else if (c == '#' && !sq && !dq && (k == 0 || std::isspace((unsigned char)s[k - 1]))) return s.substr(0, k);
    }
    return s;
  }
  static std::string trim(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
  }
  // drops a leading tag (!Rpy and the like)
  static std::string untag(const std::string& s) {
    std::string t = trim(s);
    if (!t.empty() && t[0] == '!') {
      size_t k = 0;
      while (k < t.size() && !std::isspace((unsigned char)t[k])) ++k;
      t = trim(t.substr(k));
    }
    return t;
  }
  static std::string unquote(const std::string& s) {
    if (s.size() >= 2 && ((s.front() == '"' && s.back() == '"') || (s.front() == '\'' && s.back() == '\'')))
      return s.substr(1, s.size() - 2);
    return s;
  }
  // position of the mapping colon of a "key: value" line, or npos
  static size_t key_colon(const std::string& s) {
    bool sq = false, dq = false;
    int depth = 0;
    for (size_t k = 0; k < s.size(); ++k) {
      const char c = s[k];
      if (c == '\'' && !dq) sq = !sq;
      else if (c == '"' && !sq) dq = !dq;
      else if (!sq && !dq && (c == '[' || c == '{')) ++depth;
      else if (!sq && !dq && (c == ']' || c == '}')) --depth;
      else if (c == ':' && !sq && !dq && depth == 0 && (k + 1 == s.size() || s[k + 1] == ' ')) return k;
    }
    return std::string::npos;
  }

  // flow collections: [a, b] and {k: v}
  static YNode parse_flow(const std::string& src, size_t& k) {
    auto ws = [&]() {
      while (k < src.size() && std::isspace((unsigned char)src[k])) ++k;
    };
    ws();
    if (k < src.size() && src[k] == '!') {  // tag
      while (k < src.size() && !std::isspace((unsigned char)src[k])) ++k;
      ws();
    }
    YNode n;
    if (k < src.size() && (src[k] == '[' || src[k] == '{')) {
      const bool seq = src[k] == '[';
      const char close = seq ? ']' : '}';
      n.kind = seq ? YNode::SEQ : YNode::MAP;
      ++k;
      for (;;) {
        ws();
        if (k >= src.size()) throw std::runtime_error("YAML: unterminated flow collection");
        if (src[k] == close) {
          ++k;
          return n;
        }
        if (seq) {
          n.seq.push_back(parse_flow(src, k));
        } else {
          const size_t b = k;
          while (k < src.size() && src[k] != ':') ++k;
          if (k >= src.size()) throw std::runtime_error("YAML: flow mapping without ':'");
          const std::string key = unquote(trim(src.substr(b, k - b)));
          ++k;
          n.map.emplace_back(key, parse_flow(src, k));
        }
        ws();
        if (k < src.size() && src[k] == ',') ++k;
      }
    }
    const size_t b = k;
    if (k < src.size() && (src[k] == '"' || src[k] == '\'')) {
      const char q = src[k];
      const size_t e = src.find(q, k + 1);
      if (e == std::string::npos) throw std::runtime_error("YAML: unterminated quoted scalar");
      k = e + 1;
      n.scalar = src.substr(b + 1, e - b - 1);
      return n;
    }
    while (k < src.size() && src[k] != ',' && src[k] != ']' && src[k] != '}') ++k;
    n.scalar = trim(src.substr(b, k - b));
    return n;
  }

  static YNode scalar_or_flow(const std::string& v) {
    const std::string t = untag(v);
    if (!t.empty() && (t[0] == '[' || t[0] == '{')) {
      size_t k = 0;
      return parse_flow(t, k);
    }
    YNode n;
    n.scalar = unquote(t);
    return n;
  }

  // the node made of the lines from k on at exactly `indent`
  YNode parse_block(size_t& k, int indent) {
    YNode n;
    const bool seq = lines_[k].text.rfind("- ", 0) == 0 || lines_[k].text == "-";
    n.kind = seq ? YNode::SEQ : YNode::MAP;
    while (k < lines_.size() && lines_[k].indent == indent) {
      const std::string& t = lines_[k].text;
      const bool item = t.rfind("- ", 0) == 0 || t == "-";
      if (seq && !item) break;  // a sequence written at its key's indentation ends here
      if (item != seq) throw std::runtime_error("YAML: mixed sequence and mapping on line " + std::to_string(lines_[k].no));
      if (seq) {
        const std::string rest = t == "-" ? std::string() : t.substr(2);
        size_t lead = 2;
        while (lead < t.size() && t[lead] == ' ') ++lead;
        if (trim(rest).empty()) {  // the item is the nested block below
          ++k;
          if (k < lines_.size() && lines_[k].indent > indent) n.seq.push_back(parse_block(k, lines_[k].indent));
          else n.seq.push_back(YNode{});
        } else if (key_colon(trim(rest)) != std::string::npos) {
          // "- key: value" opens a mapping whose keys sit at indent + lead
          lines_[k].indent = indent + (int)lead;
          lines_[k].text = trim(rest);
          n.seq.push_back(parse_block(k, indent + (int)lead));
        } else {
          n.seq.push_back(scalar_or_flow(rest));
          ++k;
        }
      } else {
        const size_t c = key_colon(t);
        if (c == std::string::npos) throw std::runtime_error("YAML: expected 'key: value' on line " + std::to_string(lines_[k].no));
        const std::string key = unquote(trim(t.substr(0, c)));
        const std::string val = trim(t.substr(c + 1));
        ++k;
        if (untag(val).empty()) {
          if (k < lines_.size() && lines_[k].indent > indent) n.map.emplace_back(key, parse_block(k, lines_[k].indent));
          else if (k < lines_.size() && lines_[k].indent == indent && lines_[k].text.rfind("- ", 0) == 0)
            n.map.emplace_back(key, parse_block(k, indent));  // a sequence at the key's indentation
          else n.map.emplace_back(key, YNode{});
        } else {
          n.map.emplace_back(key, scalar_or_flow(val));
        }
      }
    }
    if (k < lines_.size() && lines_[k].indent > indent)
      throw std::runtime_error("YAML: unexpected indentation on line " + std::to_string(lines_[k].no));
    return n;
  }
};

// ------------------------------------------------------------------ model
enum { J_FIXED = 0, J_REVOLUTE = 1, J_PRISMATIC = 2 };
enum { S_BOX = 0, S_SPHERE = 1, S_CYLINDER = 2, S_CAPSULE = 3 };
enum { G_ROBOT = 0, G_WORLD = 1 };

struct Mat4 {
  float m[16];  // row-major while building
};

static Mat4 identity() {
  Mat4 x{};
  x.m[0] = x.m[5] = x.m[10] = x.m[15] = 1.f;
  return x;
}

struct JointRec {
  std::string name;
  int type = J_FIXED;
  Mat4 X = identity();
  int parent = -1, child = -1;
  float axis[3] = {0, 0, 0};
  float lower = -FLT_MAX, upper = FLT_MAX;
};

struct LinkRec {
  std::string name;
  int parent_joint = -1;
  std::vector<int> child_joints;
};

struct GeomRec {
  int type = S_BOX;
  float dims[3] = {0, 0, 0};
  int link = 0;
  int group = G_ROBOT;
  Mat4 X = identity();
};

// a Python-style float: decimal string -> double -> float
static float to_f32(const std::string& s) {
  const char* b = s.c_str();
  char* e = nullptr;
  const double v = std::strtod(b, &e);
  while (e && *e && std::isspace((unsigned char)*e)) ++e;
  if (e == b || (e && *e)) throw std::runtime_error("could not convert string to float: '" + s + "'");
  return (float)v;
}

static std::vector<float> floats(const std::string& s, size_t n) {
  std::istringstream in(s);
  std::vector<float> v;
  std::string tok;
  while (in >> tok) v.push_back(to_f32(tok));
  if (v.size() < n) throw std::runtime_error("expected " + std::to_string(n) + " numbers in '" + s + "'");
  v.resize(n);
  return v;
}

// Rz(y) Ry(p) Rx(r) in double, rounded to float (urdf_parser.cpp:370-375)
static Mat4 transform(const float* rpy, const float* t) {
  const double cr = std::cos((double)rpy[0]), sr = std::sin((double)rpy[0]);
  const double cp = std::cos((double)rpy[1]), sp = std::sin((double)rpy[1]);
  const double cy = std::cos((double)rpy[2]), sy = std::sin((double)rpy[2]);
  const double rx[9] = {1, 0, 0, 0, cr, -sr, 0, sr, cr};
  const double ry[9] = {cp, 0, sp, 0, 1, 0, -sp, 0, cp};
  const double rz[9] = {cy, -sy, 0, sy, cy, 0, 0, 0, 1};
  double zy[9], r[9];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += rz[3 * i + k] * ry[3 * k + j];
      zy[3 * i + j] = s;
    }
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double s = 0;
      for (int k = 0; k < 3; ++k) s += zy[3 * i + k] * rx[3 * k + j];
      r[3 * i + j] = s;
    }
  Mat4 X = identity();
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) X.m[4 * i + j] = (float)r[3 * i + j];
    X.m[4 * i + 3] = t[i];
  }
  return X;
}

// urdf_parser.cpp:321-381
static Mat4 parse_origin(const XmlNode* el) {
  if (!el) return identity();
  const std::string* xyz = el->attr("xyz");
  if (!xyz) throw std::runtime_error("[CSDECOMP:URDFPARSER] no position specified for joint origin");
  const std::vector<float> t = floats(*xyz, 3);
  float rpy[3] = {0, 0, 0};
  if (const std::string* r = el->attr("rpy")) {
    const std::vector<float> v = floats(*r, 3);
    rpy[0] = v[0];
    rpy[1] = v[1];
    rpy[2] = v[2];
  }
  return transform(rpy, t.data());
}

static std::string req_attr(const XmlNode& el, const char* name) {
  const std::string* v = el.attr(name);
  if (!v) throw std::runtime_error("<" + el.tag + "> without attribute '" + name + "'");
  return *v;
}

class Parser {
 public:
  std::vector<LinkRec> links;
  std::vector<JointRec> joints;
  std::unordered_map<std::string, int> link_index, joint_index;
  std::vector<GeomRec> geoms;
  std::vector<std::pair<std::string, int>> geom_names;  // in insertion order
  std::unordered_map<std::string, std::string> packages;
  bool parsed = false;
  // finalized tables
  std::vector<int> cfg_idx, traversal, robot_ids, pairs;
  std::vector<float> lower, upper;
  int dim = 0;
  // csd_plant_desc_t storage
  std::vector<int32_t> d_jtype, d_jparent, d_jchild, d_gtype, d_glink, d_ggroup;
  std::vector<float> d_jX, d_jaxis, d_gdims, d_gX;

  bool register_package(const std::string& name, const std::string& path) {
    struct stat st;
    if (name.empty() || path.empty() || stat(path.c_str(), &st) != 0) return false;
    packages[name] = path;
    return true;
  }

  std::string resolve(const std::string& path) const {
    const std::string pre = "package://";
    if (path.rfind(pre, 0) == 0) {
      const std::string rest = path.substr(pre.size());
      const size_t sl = rest.find('/');
      const std::string pkg = rest.substr(0, sl);
      auto it = packages.find(pkg);
      if (it != packages.end()) {
        const std::string rel = sl == std::string::npos ? std::string() : rest.substr(sl + 1);
        std::string base = it->second;
        if (!rel.empty() && rel[0] == '/') return rel;
        if (!base.empty() && base.back() != '/') base.push_back('/');
        return base + rel;
      }
    }
    return path;
  }

  // kinematic_tree.cpp:14-28
  int add_link(const std::string& name) {
    if (link_index.count(name)) throw std::runtime_error("Duplicate link name detected in URDF. Name : " + name);
    const int idx = (int)links.size();
    links.push_back(LinkRec{name, -1, {}});
    link_index[name] = idx;
    return idx;
  }

  int get_link(const std::string& name) const {
    auto it = link_index.find(name);
    if (it == link_index.end()) throw std::runtime_error("[KinematicTree] Invalid link name " + name);
    return it->second;
  }

  // urdf_parser.cpp:280-320, 403-466 (capsules accepted)
  void parse_link(const XmlNode& el) {
    const std::string name = req_attr(el, "name");
    if (el.attr("origin")) throw std::runtime_error("Global origin tags are not supported in links");
    const int idx = add_link(name);
    int n = 0;
    for (const XmlNode& col : el.children) {
      if (col.tag != "collision") continue;
      const std::string cname = col.attr("name") ? *col.attr("name") + "::" + std::to_string(n + 1)
                                                 : name + "::col_geom::" + std::to_string(n + 1);
      GeomRec g;
      if (const XmlNode* o = col.child("origin")) g.X = parse_origin(o);
      if (const XmlNode* geo = col.child("geometry")) {
        if (geo->children.empty()) throw std::runtime_error("No valid geometry type specified.");
        const XmlNode& shape = geo->children[0];
        if (shape.tag == "box") {
          g.type = S_BOX;
          const std::vector<float> v = floats(req_attr(shape, "size"), 3);
          std::copy(v.begin(), v.end(), g.dims);
        } else if (shape.tag == "sphere") {
          g.type = S_SPHERE;
          g.dims[0] = to_f32(req_attr(shape, "radius"));
          g.dims[1] = g.dims[2] = -1.f;
        } else if (shape.tag == "cylinder") {
          throw std::runtime_error("cylider not yet implemented");
        } else if (shape.tag == "capsule") {
          g.type = S_CAPSULE;
          g.dims[0] = g.dims[2] = to_f32(req_attr(shape, "radius"));
          g.dims[1] = to_f32(req_attr(shape, "length"));
        }
      }
      g.link = idx;
      geom_names.emplace_back(cname, (int)geoms.size());
      geoms.push_back(g);
      ++n;
    }
  }

  // urdf_parser.cpp:208-278, kinematic_tree.cpp:30-52
  void parse_joint(const XmlNode& el) {
    const std::string* ts = el.attr("type");
    const std::string tstr = ts ? *ts : std::string("None");
    JointRec j;
    if (tstr == "fixed") j.type = J_FIXED;
    else if (tstr == "revolute") j.type = J_REVOLUTE;
    else if (tstr == "prismatic") j.type = J_PRISMATIC;
    else throw std::runtime_error("Unsupported joint type: " + tstr);
    if (j.type != J_FIXED) {
      const XmlNode* ax = el.child("axis");
      if (!ax) throw std::runtime_error("revolute or prismatic joint without axis");
      const std::vector<float> a = floats(req_attr(*ax, "xyz"), 3);
      const float nrm = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
      for (int k = 0; k < 3; ++k) j.axis[k] = a[k] / nrm;
    }
    const XmlNode* parent = el.child("parent");
    const XmlNode* child = el.child("child");
    if (!parent || !child) throw std::runtime_error("Joint is missing parent or child element");
    j.name = el.attr("name") ? *el.attr("name") : std::string();
    j.X = parse_origin(el.child("origin"));
    j.parent = get_link(req_attr(*parent, "link"));
    j.child = get_link(req_attr(*child, "link"));
    if (const XmlNode* lim = el.child("limit")) {
      j.lower = lim->attr("lower") ? to_f32(*lim->attr("lower")) : 0.f;
      j.upper = lim->attr("upper") ? to_f32(*lim->attr("upper")) : 0.f;
    }
    if (joint_index.count(j.name)) throw std::runtime_error("Duplicate joint name detected in URDF.");
    const int idx = (int)joints.size();
    joint_index[j.name] = idx;
    links[j.parent].child_joints.push_back(idx);
    links[j.child].parent_joint = idx;
    joints.push_back(j);
  }

  // urdf_parser.cpp:90-206
  bool parse_robot(const XmlNode& robot) {
    if (robot.tag != "robot") return false;
    add_link("world");
    for (const XmlNode& c : robot.children)
      if (c.tag == "link") parse_link(c);
    for (const XmlNode& c : robot.children)
      if (c.tag == "joint") parse_joint(c);
    bool connected = false;
    for (const JointRec& j : joints) connected |= j.parent == 0;
    if (!connected)
      throw std::runtime_error("[CSDECOMP:URDFPARSER] The provided urdf is not connected to the 'world' link");
    for (size_t l = 1; l < links.size(); ++l)
      if (links[l].parent_joint < 0)
        throw std::runtime_error("[CSDECOMP:URDFPARSER] The link " + links[l].name +
                                 " has no parent joint; every model must be connected to the world frame.");
    finalize();
    parsed = true;
    return true;
  }

  // kinematic_tree.cpp:82-146
  void finalize() {
    dim = 0;
    cfg_idx.assign(joints.size(), -1);
    for (size_t j = 0; j < joints.size(); ++j)
      if (joints[j].type != J_FIXED) cfg_idx[j] = dim++;
    traversal.clear();
    std::vector<int> stack(links[0].child_joints.begin(), links[0].child_joints.end());
    while (!stack.empty()) {
      const int j = stack.back();
      stack.pop_back();
      traversal.push_back(j);
      const auto& cj = links[joints[j].child].child_joints;
      stack.insert(stack.end(), cj.begin(), cj.end());
    }
    lower.clear();
    upper.clear();
    for (const JointRec& j : joints)
      if (j.type != J_FIXED) {
        lower.push_back(j.lower);
        upper.push_back(j.upper);
      }
    finalize_scene();
  }

  // urdf_parser.cpp:507-531: ROBOT unless the link reaches the world through fixed joints only
  void group_geometries() {
    for (GeomRec& g : geoms) {
      int pj = links[g.link].parent_joint;
      if (pj < 0) throw std::runtime_error("collision geometry attached to the world link is not supported");
      for (size_t guard = 0;; ++guard) {
        const JointRec& jt = joints[pj];
        if (jt.type != J_FIXED) {
          g.group = G_ROBOT;
          break;
        }
        if (jt.parent == 0) {
          g.group = G_WORLD;
          break;
        }
        pj = links[jt.parent].parent_joint;
        if (pj == -1 || guard > joints.size()) throw std::runtime_error("The kinematic tree appears to be disconnected.");
      }
    }
  }

  // urdf_parser.cpp:546-613: pairs (a < b) with a robot geometry, not on one
  // link, not parent/child links, not joined by fixed joints only
  void finalize_scene() {
    group_geometries();
    robot_ids.clear();
    for (size_t g = 0; g < geoms.size(); ++g)
      if (geoms[g].group == G_ROBOT) robot_ids.push_back((int)g);
    const int L = (int)links.size();
    std::vector<int> depth(L, 0);
    for (int j : traversal) depth[joints[j].child] = depth[joints[j].parent] + 1;
    auto all_fixed = [&](int a, int b) {
      bool fixed = true;
      while (a != b) {
        int j;
        if (depth[a] >= depth[b]) {
          j = links[a].parent_joint;
          a = joints[j].parent;
        } else {
          j = links[b].parent_joint;
          b = joints[j].parent;
        }
        if (joints[j].type != J_FIXED) fixed = false;
      }
      return fixed;
    };
    std::map<std::pair<int, int>, bool> fixed_memo;
    auto fixed_path = [&](int a, int b) {
      auto key = std::make_pair(a, b);
      auto it = fixed_memo.find(key);
      if (it != fixed_memo.end()) return it->second;
      const bool f = all_fixed(a, b);
      fixed_memo[key] = f;
      return f;
    };
    auto parent_of = [&](int l) { return links[l].parent_joint >= 0 ? joints[links[l].parent_joint].parent : -1; };
    pairs.clear();
    const int G = (int)geoms.size();
    for (int a = 0; a < G; ++a)
      for (int b = a + 1; b < G; ++b) {
        const GeomRec& ga = geoms[a];
        const GeomRec& gb = geoms[b];
        if (ga.group == G_WORLD && gb.group == G_WORLD) continue;
        if (parent_of(ga.link) == gb.link || parent_of(gb.link) == ga.link) continue;
        if (ga.link == gb.link) continue;
        if (fixed_path(ga.link, gb.link)) continue;
        pairs.push_back(a);
        pairs.push_back(b);
      }
    build_desc();
  }

  void build_desc() {
    const size_t J = joints.size(), G = geoms.size();
    d_jtype.resize(J);
    d_jparent.resize(J);
    d_jchild.resize(J);
    d_jX.resize(16 * J);
    d_jaxis.resize(3 * J);
    for (size_t j = 0; j < J; ++j) {
      d_jtype[j] = joints[j].type;
      d_jparent[j] = joints[j].parent;
      d_jchild[j] = joints[j].child;
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) d_jX[16 * j + 4 * c + r] = joints[j].X.m[4 * r + c];  // column-major
      for (int k = 0; k < 3; ++k) d_jaxis[3 * j + k] = joints[j].axis[k];
    }
    d_gtype.resize(G);
    d_glink.resize(G);
    d_ggroup.resize(G);
    d_gdims.resize(3 * G);
    d_gX.resize(16 * G);
    for (size_t g = 0; g < G; ++g) {
      d_gtype[g] = geoms[g].type;
      d_glink[g] = geoms[g].link;
      d_ggroup[g] = geoms[g].group;
      for (int k = 0; k < 3; ++k) d_gdims[3 * g + k] = geoms[g].dims[k];
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) d_gX[16 * g + 4 * c + r] = geoms[g].X.m[4 * r + c];
    }
  }

  // ---- directives, urdf_parser.cpp:618-778
  void rename(XmlNode& el, const std::string& prefix) {
    if (const std::string* n = el.attr("name")) el.set_attr("name", prefix + "::" + *n);
    if (el.tag == "joint") {
      for (XmlNode& c : el.children) {
        if (c.tag != "parent" && c.tag != "child") continue;
        const std::string* l = c.attr("link");
        if (!l) continue;
        if (c.tag == "parent" && *l == "world")
          throw std::runtime_error("Directly specifying the world link as parent is not supported");
        c.set_attr("link", prefix + "::" + *l);
      }
    }
    for (XmlNode& c : el.children) rename(c, prefix);
  }

  static std::string scalar(const YNode* n, const char* what) {
    if (!n || n->kind != YNode::SCALAR) throw std::runtime_error(std::string("directive field '") + what + "' missing");
    return n->scalar;
  }

  static std::string fmt6g(double v) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.6g", v);
    return buf;
  }

  XmlNode directives_to_robot(const std::string& path) {
    std::ifstream f(path);
    if (!f) throw std::runtime_error("Failed to open directives file: " + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const YNode doc = YamlReader(ss.str()).parse();
    const YNode* dirs = doc.get("directives");
    if (!dirs || dirs->kind != YNode::SEQ) throw std::runtime_error("directives file without a 'directives' list");
    XmlNode robot;
    robot.tag = "robot";
    robot.attrs.emplace_back("name", "combined_robot");
    for (const YNode& d : dirs->seq) {
      if (const YNode* m = d.get("add_model")) {
        const std::string name = scalar(m->get("name"), "name");
        const std::string file = resolve(scalar(m->get("file"), "file"));
        std::ifstream mf(file);
        if (!mf) throw std::runtime_error("Failed to load URDF file: " + file);
        std::stringstream ms;
        ms << mf.rdbuf();
        const std::string text = ms.str();
        XmlNode root = XmlReader(text).parse_document();
        rename(root, name);
        for (XmlNode& c : root.children) robot.children.push_back(std::move(c));
      } else if (const YNode* w = d.get("add_weld")) {
        const std::string p = scalar(w->get("parent"), "parent"), c = scalar(w->get("child"), "child");
        XmlNode j;
        j.tag = "joint";
        j.attrs = {{"name", "weld_" + p + "_to_" + c}, {"type", "fixed"}};
        XmlNode pe, ce;
        pe.tag = "parent";
        pe.attrs = {{"link", p}};
        ce.tag = "child";
        ce.attrs = {{"link", c}};
        j.children = {pe, ce};
        robot.children.push_back(j);
      } else if (const YNode* fr = d.get("add_frame")) {
        const std::string name = scalar(fr->get("name"), "name");
        const YNode* X = fr->get("X_PF");
        if (!X) throw std::runtime_error("add_frame without X_PF");
        const std::string base = scalar(X->get("base_frame"), "base_frame");
        const YNode* tr = X->get("translation");
        const YNode* rot = X->get("rotation");
        const YNode* deg = rot ? rot->get("deg") : nullptr;
        if (!tr || tr->kind != YNode::SEQ || tr->seq.size() != 3 || !deg || deg->kind != YNode::SEQ || deg->seq.size() != 3)
          throw std::runtime_error("add_frame needs translation [x, y, z] and rotation deg [r, p, y]");
        double t[3], rpy[3];
        for (int k = 0; k < 3; ++k) {
          t[k] = std::strtod(tr->seq[k].scalar.c_str(), nullptr);
          rpy[k] = std::strtod(deg->seq[k].scalar.c_str(), nullptr) * M_PI / 180.0;
        }
        XmlNode link;
        link.tag = "link";
        link.attrs = {{"name", name}};
        robot.children.push_back(link);
        XmlNode j, pe, ce, o;
        j.tag = "joint";
        j.attrs = {{"name", base + "_to_" + name}, {"type", "fixed"}};
        pe.tag = "parent";
        pe.attrs = {{"link", base}};
        ce.tag = "child";
        ce.attrs = {{"link", name}};
        o.tag = "origin";
        o.attrs = {{"xyz", fmt6g(t[0]) + " " + fmt6g(t[1]) + " " + fmt6g(t[2])},
                   {"rpy", fmt6g(rpy[0]) + " " + fmt6g(rpy[1]) + " " + fmt6g(rpy[2])}};
        j.children = {pe, ce, o};
        robot.children.push_back(j);
      }
    }
    return robot;
  }
};

}  // namespace urdf
}  // namespace csd

struct csd_urdf_s {
  csd::urdf::Parser p;
};

using namespace csd;

#define CSD_URDF_TRY(body)                                           \
  try {                                                              \
    body;                                                            \
  } catch (const std::exception& e) {                                \
    set_error(e.what());                                             \
    return CSD_ERR_INVALID;                                          \
  } catch (...) {                                                    \
    set_error("unknown error while loading the model");              \
    return CSD_ERR_INVALID;                                          \
  }

extern "C" {

csd_status_t csd_urdf_create(csd_urdf_t* out) {
  CSD_CHECK(out, CSD_ERR_INVALID, "null argument");
  *out = new (std::nothrow) csd_urdf_s();
  CSD_CHECK(*out, CSD_ERR_CAPACITY, "out of host memory");
  return CSD_OK;
}

csd_status_t csd_urdf_destroy(csd_urdf_t h) {
  delete h;
  return CSD_OK;
}

csd_status_t csd_urdf_register_package(csd_urdf_t h, const char* name, const char* path, int32_t* registered) {
  CSD_CHECK(h && name && path, CSD_ERR_INVALID, "null argument");
  const bool ok = h->p.register_package(name, path);
  if (registered) *registered = ok ? 1 : 0;
  return CSD_OK;
}

csd_status_t csd_urdf_parse_string(csd_urdf_t h, const char* text) {
  CSD_CHECK(h && text, CSD_ERR_INVALID, "null argument");
  CSD_URDF_TRY({
    const std::string s(text);
    const urdf::XmlNode root = urdf::XmlReader(s).parse_document();
    if (!h->p.parse_robot(root)) {
      set_error("Root element is not 'robot'");
      return CSD_ERR_INVALID;
    }
  });
  return CSD_OK;
}

csd_status_t csd_urdf_parse_file(csd_urdf_t h, const char* path) {
  CSD_CHECK(h && path, CSD_ERR_INVALID, "null argument");
  std::ifstream f(path);
  if (!f) {
    set_error(std::string("Failed to load URDF file: ") + path);
    return CSD_ERR_INVALID;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();
  return csd_urdf_parse_string(h, text.c_str());
}

csd_status_t csd_urdf_parse_directives(csd_urdf_t h, const char* path) {
  CSD_CHECK(h && path, CSD_ERR_INVALID, "null argument");
  CSD_URDF_TRY({
    const urdf::XmlNode robot = h->p.directives_to_robot(path);
    h->p.parse_robot(robot);
  });
  return CSD_OK;
}

csd_status_t csd_urdf_plant_desc(csd_urdf_t h, csd_plant_desc_t* d) {
  CSD_CHECK(h && d, CSD_ERR_INVALID, "null argument");
  CSD_CHECK(h->p.parsed, CSD_ERR_INVALID, "No URDF has been parsed yet");
  urdf::Parser& p = h->p;
  d->num_joints = (int32_t)p.joints.size();
  d->num_links = (int32_t)p.links.size();
  d->num_configuration_variables = p.dim;
  d->num_geometries = (int32_t)p.geoms.size();
  d->num_collision_pairs = (int32_t)(p.pairs.size() / 2);
  d->joint_type = p.d_jtype.data();
  d->joint_parent_link = p.d_jparent.data();
  d->joint_child_link = p.d_jchild.data();
  d->joint_idx_to_config_idx = p.cfg_idx.data();
  d->joint_traversal_sequence = p.traversal.data();
  d->joint_X_PL_J = p.d_jX.data();
  d->joint_axis = p.d_jaxis.data();
  d->geom_type = p.d_gtype.data();
  d->geom_link_index = p.d_glink.data();
  d->geom_group = p.d_ggroup.data();
  d->geom_dimensions = p.d_gdims.data();
  d->geom_X_L_B = p.d_gX.data();
  d->collision_pairs_flat = p.pairs.data();
  return CSD_OK;
}

csd_status_t csd_urdf_limits(csd_urdf_t h, float* lower, float* upper) {
  CSD_CHECK(h && lower && upper, CSD_ERR_INVALID, "null argument");
  CSD_CHECK(h->p.parsed, CSD_ERR_INVALID, "No URDF has been parsed yet");
  std::copy(h->p.lower.begin(), h->p.lower.end(), lower);
  std::copy(h->p.upper.begin(), h->p.upper.end(), upper);
  return CSD_OK;
}

csd_status_t csd_urdf_robot_geometry_ids(csd_urdf_t h, const int32_t** ids, int32_t* n) {
  CSD_CHECK(h && ids && n, CSD_ERR_INVALID, "null argument");
  CSD_CHECK(h->p.parsed, CSD_ERR_INVALID, "No URDF has been parsed yet");
  *ids = h->p.robot_ids.data();
  *n = (int32_t)h->p.robot_ids.size();
  return CSD_OK;
}

csd_status_t csd_urdf_link_index(csd_urdf_t h, const char* name, int32_t* index) {
  CSD_CHECK(h && name && index, CSD_ERR_INVALID, "null argument");
  auto it = h->p.link_index.find(name);
  CSD_CHECK(it != h->p.link_index.end(), CSD_ERR_INVALID, std::string("[KinematicTree] Invalid link name ") + name);
  *index = it->second;
  return CSD_OK;
}

csd_status_t csd_urdf_geometry_index(csd_urdf_t h, const char* name, int32_t* index) {
  CSD_CHECK(h && name && index, CSD_ERR_INVALID, "null argument");
  for (auto it = h->p.geom_names.rbegin(); it != h->p.geom_names.rend(); ++it)  // a repeated name: the last one
    if (it->first == name) {
      *index = it->second;
      return CSD_OK;
    }
  set_error(std::string("no collision geometry named ") + name);
  return CSD_ERR_INVALID;
}

}  // extern "C"
