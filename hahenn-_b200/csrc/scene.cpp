// Minimal JSON reader and the scene model (see scene.h).
#include "scene.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace suiri {

const JVal* JVal::get(const char* key) const {
  if (kind != Obj) return nullptr;
  for (const auto& kv : obj)
    if (kv.first == key) return &kv.second;
  return nullptr;
}

namespace {

struct Parser {
  const char* p;
  const char* end;
  std::string err;
  int depth = 0;

  void ws() {
    while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
  }
  bool fail(const char* m) {
    if (err.empty()) err = m;
    return false;
  }
  bool lit(const char* w) {
    const size_t n = strlen(w);
    if ((size_t)(end - p) < n || strncmp(p, w, n) != 0) return fail("bad literal");
    p += n;
    return true;
  }
  bool str(std::string& out) {
    if (p >= end || *p != '"') return fail("expected string");
    ++p;
    while (p < end && *p != '"') {
      if (*p == '\\') {
        ++p;
        if (p >= end) return fail("bad escape");
        switch (*p) {
          case '"': out += '"'; break;
          case '\\': out += '\\'; break;
          case '/': out += '/'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'n': out += '\n'; break;
          case 'r': out += '\r'; break;
          case 't': out += '\t'; break;
          case 'u': {
            if (end - p < 5) return fail("bad \\u escape");
            unsigned cp = (unsigned)strtoul(std::string(p + 1, p + 5).c_str(), nullptr, 16);
            p += 4;
            if (cp < 0x80) out += (char)cp;
            else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
            else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F)); }
            break;
          }
          default: return fail("bad escape");
        }
        ++p;
      } else {
        out += *p++;
      }
    }
    if (p >= end) return fail("unterminated string");
    ++p;
    return true;
  }
  bool val(JVal& v) {
    if (++depth > 64) return fail("nesting too deep");
    ws();
    if (p >= end) return fail("unexpected end");
    bool ok = true;
    if (*p == '{') {
      v.kind = JVal::Obj;
      ++p; ws();
      if (p < end && *p == '}') { ++p; --depth; return true; }
      while (ok) {
        ws();
        std::string k;
        if (!str(k)) return false;
        ws();
        if (p >= end || *p != ':') return fail("expected ':'");
        ++p;
        JVal c;
        if (!val(c)) return false;
        v.obj.emplace_back(std::move(k), std::move(c));
        ws();
        if (p < end && *p == ',') { ++p; continue; }
        if (p < end && *p == '}') { ++p; break; }
        return fail("expected ',' or '}'");
      }
    } else if (*p == '[') {
      v.kind = JVal::Arr;
      ++p; ws();
      if (p < end && *p == ']') { ++p; --depth; return true; }
      while (ok) {
        JVal c;
        if (!val(c)) return false;
        v.arr.push_back(std::move(c));
        ws();
        if (p < end && *p == ',') { ++p; continue; }
        if (p < end && *p == ']') { ++p; break; }
        return fail("expected ',' or ']'");
      }
    } else if (*p == '"') {
      v.kind = JVal::Str;
      if (!str(v.s)) return false;
    } else if (*p == 't') {
      v.kind = JVal::Bool; v.b = true; if (!lit("true")) return false;
    } else if (*p == 'f') {
      v.kind = JVal::Bool; v.b = false; if (!lit("false")) return false;
    } else if (*p == 'n') {
      v.kind = JVal::Null; if (!lit("null")) return false;
    } else {
      char* e = nullptr;
      const std::string tmp(p, (size_t)std::min<ptrdiff_t>(end - p, 64));
      const double d = strtod(tmp.c_str(), &e);
      if (e == tmp.c_str()) return fail("bad value");
      v.kind = JVal::Num; v.num = d;
      p += (e - tmp.c_str());
    }
    --depth;
    return true;
  }
};

double num_or(const JVal* v, double d) { return v && v->kind == JVal::Num && std::isfinite(v->num) ? v->num : d; }

void vec_or(const JVal* v, double out[3], const double d[3]) {
  if (v && v->kind == JVal::Arr && v->arr.size() == 3 && v->arr[0].is_num() && v->arr[1].is_num() && v->arr[2].is_num() &&
      std::isfinite(v->arr[0].num) && std::isfinite(v->arr[1].num) && std::isfinite(v->arr[2].num)) {
    for (int a = 0; a < 3; ++a) out[a] = v->arr[a].num;
  } else {
    for (int a = 0; a < 3; ++a) out[a] = d[a];
  }
}

struct ShapeDef { const char* name; int type; const char* keys[4]; double dflt[4]; };
// shape table with the defaults of a fresh obstacle (src/js/10-scene.js:5-15)
const ShapeDef kShapes[] = {
    {"box", 0, {"w", "h", "d", nullptr}, {0.10, 0.06, 0.08, 0}},
    {"plate", 0, {"w", "d", "t", nullptr}, {0.22, 0.10, 0.012, 0}},
    {"sphere", 1, {"r", nullptr, nullptr, nullptr}, {0.035, 0, 0, 0}},
    {"cylinder", 2, {"r", "h", nullptr, nullptr}, {0.025, 0.12, 0, 0}},
    {"cone", 3, {"r", "h", nullptr, nullptr}, {0.04, 0.08, 0, 0}},
    {"torus", 4, {"R", "r", nullptr, nullptr}, {0.05, 0.014, 0, 0}},
    {"cup", 5, {"r", "h", "t", nullptr}, {0.04, 0.10, 0.006, 0}},
    {"container", 6, {"w", "h", "d", "t"}, {0.14, 0.06, 0.10, 0.008}},
    {"gutter", 7, {"len", "r", "t", nullptr}, {0.28, 0.03, 0.006, 0}},
};

const ShapeDef* find_shape(const std::string& s) {
  for (const auto& d : kShapes)
    if (s == d.name) return &d;
  return nullptr;
}

double dim(const ShapeDef* sd, const JVal* dims, const char* key) {
  for (int i = 0; i < 4; ++i)
    if (sd->keys[i] && strcmp(sd->keys[i], key) == 0) return num_or(dims ? dims->get(key) : nullptr, sd->dflt[i]);
  return 0.0;
}

}  // namespace

bool json_parse(const std::string& text, JVal& out, std::string& err) {
  Parser ps{text.data(), text.data() + text.size(), {}};
  if (!ps.val(out)) { err = "scene JSON: " + ps.err; return false; }
  ps.ws();
  if (ps.p != ps.end) { err = "scene JSON: trailing characters"; return false; }
  return true;
}

void euler_deg(double rx, double ry, double rz, double R[9]) {
  // R = Rz·Ry·Rx, degrees (src/js/00-util.js:22-30)
  const double d = M_PI / 180.0;
  const double cx = cos(rx * d), sx = sin(rx * d), cy = cos(ry * d), sy = sin(ry * d), cz = cos(rz * d), sz = sin(rz * d);
  const double M[9] = {cz * cy, cz * sy * sx - sz * cx, cz * sy * cx + sz * sx,
                       sz * cy, sz * sy * sx + cz * cx, sz * sy * cx - cz * sx,
                       -sy, cy * sx, cy * cx};
  memcpy(R, M, sizeof(M));
}

bool shape_params(const std::string& shape, const JVal* dims, int& type, double d[4]) {
  const ShapeDef* sd = find_shape(shape);
  if (!sd) return false;
  type = sd->type;
  d[0] = d[1] = d[2] = d[3] = 0.0;
  if (shape == "box") {
    const double w = dim(sd, dims, "w"), h = dim(sd, dims, "h"), dd = dim(sd, dims, "d");
    d[0] = w / 2; d[1] = h / 2; d[2] = dd / 2; d[3] = std::min(std::min(0.003, w / 4), std::min(h / 4, dd / 4));
  } else if (shape == "plate") {
    const double w = dim(sd, dims, "w"), t = dim(sd, dims, "t"), dd = dim(sd, dims, "d");
    d[0] = w / 2; d[1] = t / 2; d[2] = dd / 2; d[3] = std::min(0.002, t / 4);
  } else if (shape == "sphere") {
    d[0] = dim(sd, dims, "r");
  } else if (shape == "cylinder" || shape == "cone") {
    d[0] = dim(sd, dims, "r"); d[1] = dim(sd, dims, "h") / 2;
  } else if (shape == "torus") {
    d[0] = dim(sd, dims, "R"); d[1] = dim(sd, dims, "r");
  } else if (shape == "cup") {
    const double r = dim(sd, dims, "r");
    d[0] = r; d[1] = dim(sd, dims, "h") / 2; d[2] = std::min(dim(sd, dims, "t"), r * 0.8);
  } else if (shape == "container") {
    const double w = dim(sd, dims, "w"), h = dim(sd, dims, "h"), dd = dim(sd, dims, "d"), t = dim(sd, dims, "t");
    d[0] = w / 2; d[1] = h / 2; d[2] = dd / 2; d[3] = std::min(std::min(t, w / 3), std::min(dd / 3, h * 0.8));
  } else if (shape == "gutter") {
    d[0] = dim(sd, dims, "len") / 2; d[1] = dim(sd, dims, "r"); d[2] = dim(sd, dims, "t");
  }
  return true;
}

double bound_radius(int t, const double d[4]) {
  // src/js/10-scene.js:177-188
  const double a = d[0], b = d[1], c = d[2];
  switch (t) {
    case 0: case 6: return sqrt(a * a + b * b + c * c);
    case 1: return a;
    case 2: case 3: case 5: return sqrt(a * a + b * b);
    case 4: return a + b;
    case 7: return sqrt(a * a + (b + c) * (b + c));
  }
  return 0.1;
}

namespace {

// JSON text of the validated scene (the reference's validScene result, src/js/80-ui.js:430-459)
std::string jnum(double v) {
  char b[40];
  snprintf(b, sizeof b, "%.15g", v);
  if (strtod(b, nullptr) != v) snprintf(b, sizeof b, "%.17g", v);
  return b;
}
std::string jstr(const std::string& v) {
  std::string o = "\"";
  for (const char c : v) {
    if (c == '"' || c == '\\') { o += '\\'; o += c; }
    else if ((unsigned char)c < 0x20) { char b[8]; snprintf(b, sizeof b, "\\u%04x", (unsigned)(unsigned char)c); o += b; }
    else o += c;
  }
  return o + "\"";
}
std::string jvec(const double v[3]) { return "[" + jnum(v[0]) + "," + jnum(v[1]) + "," + jnum(v[2]) + "]"; }

// a string field: the item's if it is a non-empty string, else the fresh item's
std::string str_or(const JVal* v, const char* d) { return v && v->kind == JVal::Str && !v->s.empty() ? v->s : std::string(d); }
bool bool_or(const JVal* v, bool d) { return v && v->kind == JVal::Bool ? v->b : d; }

// names, colours and materials of fresh items (src/js/10-scene.js:5-15, :56-86)
const char* shape_label(const std::string& s) {
  static const char* const L[][2] = {{"box", "箱"}, {"plate", "板"}, {"sphere", "球"}, {"cylinder", "円柱"}, {"cone", "円錐"},
                                     {"torus", "ドーナツ"}, {"cup", "コップ"}, {"container", "容器"}, {"gutter", "樋（とい）"}};
  for (const auto& x : L)
    if (s == x[0]) return x[1];
  return "箱";
}
bool is_material(const std::string& m) { return m == "ceramic" || m == "plastic" || m == "metal" || m == "stone"; }

}  // namespace

bool parse_items(const JVal& items, Scene& sc, std::string& err) {
  if (items.kind != JVal::Arr) { err = "scene JSON: items must be an array"; return false; }
  // ids as validScene assigns them: a positive integer not seen before is kept; the others get max + 1, +2, …
  // in item order
  std::vector<const JVal*> kept;
  std::vector<long long> ids;
  std::vector<long long> seen;
  for (const JVal& it : items.arr) {
    if (it.kind != JVal::Obj) continue;
    const JVal* kind = it.get("kind");
    if (!kind || kind->kind != JVal::Str) continue;
    if (kind->s != "obstacle" && kind->s != "drain" && kind->s != "block" && kind->s != "source") continue;
    const JVal* idv = it.get("id");
    long long id = -1;
    if (idv && idv->is_num() && idv->num > 0 && idv->num == floor(idv->num) && idv->num < 2147483647.0 &&
        std::find(seen.begin(), seen.end(), (long long)idv->num) == seen.end()) {
      id = (long long)idv->num;
      seen.push_back(id);
    }
    kept.push_back(&it);
    ids.push_back(id);
  }
  long long next = 1;
  for (long long v : seen) next = std::max(next, v + 1);
  for (long long& v : ids)
    if (v < 0) v = next++;
  std::string out = "[";
  for (size_t n = 0; n < kept.size(); ++n) {
    const JVal& it = *kept[n];
    const std::string kind = it.get("kind")->s;
    const int id = (int)ids[n];
    std::string js = "{\"id\":" + std::to_string(id) + ",\"kind\":" + jstr(kind);
    if (kind == "obstacle" || kind == "drain") {
      SceneItem si;
      si.id = id;
      Obj& o = si.obj;
      memset(&o, 0, sizeof(o));
      const double zero[3] = {0, 0, 0};
      double rot[3];
      vec_or(it.get("rot"), rot, zero);
      euler_deg(rot[0], rot[1], rot[2], si.R);
      memcpy(o.rot, si.R, sizeof(si.R));
      if (kind == "obstacle") {
        const double p0[3] = {0, 0.05, 0};
        vec_or(it.get("pos"), o.pos, p0);
        const JVal* sh = it.get("shape");
        const std::string shape = (sh && sh->kind == JVal::Str && find_shape(sh->s)) ? sh->s : "box";
        shape_params(shape, it.get("dims"), o.type, o.dims);
        o.bound = bound_radius(o.type, o.dims) + 0.002;
        o.flag = 1;
        const ShapeDef* sd = find_shape(shape);
        const JVal* dims = it.get("dims");
        std::string dj = "{";
        for (int k = 0; k < 4 && sd->keys[k]; ++k)
          dj += std::string(k ? "," : "") + jstr(sd->keys[k]) + ":" + jnum(dim(sd, dims, sd->keys[k]));
        dj += "}";
        const char* color = shape == "cup" ? "#e9e4da" : shape == "gutter" ? "#8a8f94" : "#c9c2b4";
        const char* mat = shape == "gutter" ? "metal" : (shape == "sphere" || shape == "cone") ? "stone" : "ceramic";
        std::string m = str_or(it.get("material"), mat);
        if (!is_material(m)) m = mat;
        js += ",\"shape\":" + jstr(shape) + ",\"name\":" + jstr(str_or(it.get("name"), shape_label(shape))) +
              ",\"pos\":" + jvec(o.pos) + ",\"rot\":" + jvec(rot) + ",\"dims\":" + dj +
              ",\"color\":" + jstr(str_or(it.get("color"), color)) + ",\"material\":" + jstr(m);
      } else {
        vec_or(it.get("pos"), o.pos, zero);
        o.type = 9;
        o.dims[0] = num_or(it.get("r"), 0.025);
        o.dims[1] = 0.012;
        o.bound = o.dims[0] + 0.02;
        o.flag = 2;
        js += ",\"name\":" + jstr(str_or(it.get("name"), "排水口")) + ",\"pos\":" + jvec(o.pos) + ",\"rot\":" + jvec(rot) +
              ",\"r\":" + jnum(o.dims[0]);
      }
      sc.solids.push_back(si);
    } else if (kind == "block") {
      const double p0[3] = {0, 0.05, 0};
      double pos[3];
      vec_or(it.get("pos"), pos, p0);
      const JVal* dims = it.get("dims");
      const double w = num_or(dims ? dims->get("w") : nullptr, 0.16), h = num_or(dims ? dims->get("h") : nullptr, 0.10),
                   d = num_or(dims ? dims->get("d") : nullptr, 0.16);
      WaterBlock b;
      b.lo[0] = pos[0] - w / 2; b.lo[1] = pos[1] - h / 2; b.lo[2] = pos[2] - d / 2;
      b.hi[0] = pos[0] + w / 2; b.hi[1] = pos[1] + h / 2; b.hi[2] = pos[2] + d / 2;
      sc.blocks.push_back(b);
      js += ",\"name\":" + jstr(str_or(it.get("name"), "水の塊")) + ",\"pos\":" + jvec(pos) +
            ",\"dims\":{\"w\":" + jnum(w) + ",\"h\":" + jnum(h) + ",\"d\":" + jnum(d) + "}";
    } else {
      SourceItem s;
      s.id = id;
      const JVal* m = it.get("mode");
      if (m && m->kind == JVal::Str && (m->s == "stream" || m->s == "drops" || m->s == "shower" || m->s == "burst" || m->s == "rain"))
        s.mode = m->s;
      s.enabled = bool_or(it.get("enabled"), true);
      const double p0[3] = {0, 0.4, 0};
      vec_or(it.get("pos"), s.pos, p0);
      s.pitch = num_or(it.get("pitch"), -90); s.yaw = num_or(it.get("yaw"), 0);
      s.flow = num_or(it.get("flow"), 3.0); s.speed = num_or(it.get("speed"), 0.6);
      s.drop_d = num_or(it.get("dropD"), 5); s.drop_rate = num_or(it.get("dropRate"), 3);
      s.spread = num_or(it.get("spread"), 18); s.burst = num_or(it.get("burst"), 0.5);
      s.burst_every = num_or(it.get("burstEvery"), 0); s.rain_rate = num_or(it.get("rainRate"), 60);
      s.rain_size = num_or(it.get("rainSize"), 0.3); s.total = num_or(it.get("total"), 0);
      sc.sources.push_back(s);
      js += ",\"name\":" + jstr(str_or(it.get("name"), "水源")) + ",\"pos\":" + jvec(s.pos) + ",\"pitch\":" + jnum(s.pitch) +
            ",\"yaw\":" + jnum(s.yaw) + ",\"mode\":" + jstr(s.mode) + ",\"enabled\":" + (s.enabled ? "true" : "false") +
            ",\"flow\":" + jnum(s.flow) + ",\"speed\":" + jnum(s.speed) + ",\"dropD\":" + jnum(s.drop_d) +
            ",\"dropRate\":" + jnum(s.drop_rate) + ",\"spread\":" + jnum(s.spread) + ",\"burst\":" + jnum(s.burst) +
            ",\"burstEvery\":" + jnum(s.burst_every) + ",\"rainRate\":" + jnum(s.rain_rate) +
            ",\"rainSize\":" + jnum(s.rain_size) + ",\"total\":" + jnum(s.total);
    }
    out += (n ? "," : "") + js + "}";
  }
  sc.items_json = out + "]";
  return true;
}

bool parse_scene(const std::string& text, bool clamp_tank, Scene& sc, std::string& err) {
  JVal root;
  if (!json_parse(text, root, err)) return false;
  const JVal* s = root.get("scene");
  if (!s) s = &root;
  const JVal* tank = s->get("tank");
  const JVal* items = s->get("items");
  if (!tank || tank->kind != JVal::Obj || !items || items->kind != JVal::Arr) {
    err = "scene JSON: needs scene.tank {w,h,d} and scene.items []";
    return false;
  }
  const char* keys[3] = {"w", "h", "d"};
  for (int a = 0; a < 3; ++a) {
    const JVal* v = tank->get(keys[a]);
    if (!v || !v->is_num() || !std::isfinite(v->num) || !(v->num > 0)) {
      err = std::string("scene JSON: tank.") + keys[a] + " must be a positive number";
      return false;
    }
    sc.tank[a] = v->num;
  }
  if (clamp_tank) {
    sc.tank[0] = std::min(std::max(sc.tank[0], 0.2), 1.2);
    sc.tank[1] = std::min(std::max(sc.tank[1], 0.1), 0.6);
    sc.tank[2] = std::min(std::max(sc.tank[2], 0.15), 1.0);
  }
  return parse_items(*items, sc, err);
}

std::string scene_json_text(const Scene& sc) {
  return "{\"tank\":{\"w\":" + jnum(sc.tank[0]) + ",\"h\":" + jnum(sc.tank[1]) + ",\"d\":" + jnum(sc.tank[2]) +
         "},\"items\":" + sc.items_json + "}";
}

}  // namespace suiri
