// Scene files, configuration, task lists and float32 scene geometry.
// Compiled with -ffp-contract=off: the geometry must equal the reference's
// host computation bit for bit (see scene.h).
#include "scene.h"
#include "helio_geom.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>

#include "vecmath.h"

namespace qm {

namespace {

struct ParseError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// ---------------------------------------------------------------------------
// .scn grammar D(R(GH+)+)+ as a five-state machine
// (Tool/FileLoader/RegularExpressionTree.cpp:47-71).
enum class St { Start, Ground, Receiver, Grid, Helio };

St step(St s, char c) {
  switch (s) {
    case St::Start:
      if (c == 'D') return St::Ground;
      break;
    case St::Ground:
      if (c == 'R') return St::Receiver;
      break;
    case St::Receiver:
      if (c == 'G') return St::Grid;
      break;
    case St::Grid:
      if (c == 'H') return St::Helio;
      break;
    case St::Helio:
      if (c == 'R') return St::Receiver;
      if (c == 'G') return St::Grid;
      if (c == 'H') return St::Helio;
      break;
  }
  throw std::runtime_error("Cannot step forward.");
}

void expect_key(std::istream& in, const char* key) {
  std::string head;
  in >> head;
  if (head != key) throw std::runtime_error(std::string("Miss ' ") + key + " ' property.\n");
}

int int_field(std::istream& in, const char* key) {
  expect_key(in, key);
  int v = 0;
  in >> v;
  return v;
}

float3 float3_field(std::istream& in, const char* key) {
  expect_key(in, key);
  float3 v{0.f, 0.f, 0.f};
  in >> v.x >> v.y >> v.z;
  return v;
}

// ---------------------------------------------------------------------------
// Minimal JSON reader: enough of the format for the configuration files
// (objects, arrays, numbers, strings, true/false/null).
struct JVal {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  double num = 0.0;
  bool num_is_int = false;
  long long inum = 0;
  bool b = false;
  std::string str;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
};

struct JParser {
  const std::string& s;
  size_t i = 0;
  explicit JParser(const std::string& text) : s(text) {}
  [[noreturn]] void fail(const char* what) {
    throw ParseError(std::string("invalid JSON: ") + what + " at offset " + std::to_string(i));
  }
  void ws() {
    while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
  }
  JVal value() {
    ws();
    if (i >= s.size()) fail("unexpected end");
    char c = s[i];
    if (c == '{') return object();
    if (c == '[') return array();
    if (c == '"') {
      JVal v;
      v.kind = JVal::Str;
      v.str = string();
      return v;
    }
    if (c == 't' || c == 'f' || c == 'n') return literal();
    if (c == '-' || (c >= '0' && c <= '9')) return number();
    fail("unexpected character");
  }
  JVal literal() {
    JVal v;
    if (s.compare(i, 4, "true") == 0) {
      v.kind = JVal::Bool;
      v.b = true;
      i += 4;
    } else if (s.compare(i, 5, "false") == 0) {
      v.kind = JVal::Bool;
      i += 5;
    } else if (s.compare(i, 4, "null") == 0) {
      i += 4;
    } else {
      fail("bad literal");
    }
    return v;
  }
  JVal number() {
    size_t start = i;
    bool is_int = true;
    if (s[i] == '-') ++i;
    if (i >= s.size() || !(s[i] >= '0' && s[i] <= '9')) fail("bad number");
    while (i < s.size() && s[i] >= '0' && s[i] <= '9') ++i;
    if (i < s.size() && s[i] == '.') {
      is_int = false;
      ++i;
      if (i >= s.size() || !(s[i] >= '0' && s[i] <= '9')) fail("bad fraction");
      while (i < s.size() && s[i] >= '0' && s[i] <= '9') ++i;
    }
    if (i < s.size() && (s[i] == 'e' || s[i] == 'E')) {
      is_int = false;
      ++i;
      if (i < s.size() && (s[i] == '+' || s[i] == '-')) ++i;
      if (i >= s.size() || !(s[i] >= '0' && s[i] <= '9')) fail("bad exponent");
      while (i < s.size() && s[i] >= '0' && s[i] <= '9') ++i;
    }
    std::string tok = s.substr(start, i - start);
    JVal v;
    v.kind = JVal::Num;
    v.num = std::strtod(tok.c_str(), nullptr);
    v.num_is_int = is_int;
    if (is_int) v.inum = std::strtoll(tok.c_str(), nullptr, 10);
    return v;
  }
  std::string string() {
    if (s[i] != '"') fail("expected string");
    ++i;
    std::string out;
    while (i < s.size() && s[i] != '"') {
      if (s[i] == '\\') {
        ++i;
        if (i >= s.size()) fail("bad escape");
        char e = s[i];
        out.push_back(e == 'n' ? '\n' : e == 't' ? '\t' : e);
        ++i;
      } else {
        out.push_back(s[i++]);
      }
    }
    if (i >= s.size()) fail("unterminated string");
    ++i;
    return out;
  }
  JVal array() {
    JVal v;
    v.kind = JVal::Arr;
    ++i;
    ws();
    if (i < s.size() && s[i] == ']') {
      ++i;
      return v;
    }
    for (;;) {
      v.arr.push_back(value());
      ws();
      if (i < s.size() && s[i] == ',') {
        ++i;
        continue;
      }
      if (i < s.size() && s[i] == ']') {
        ++i;
        return v;
      }
      fail("expected , or ]");
    }
  }
  JVal object() {
    JVal v;
    v.kind = JVal::Obj;
    ++i;
    ws();
    if (i < s.size() && s[i] == '}') {
      ++i;
      return v;
    }
    for (;;) {
      ws();
      std::string key = string();
      ws();
      if (i >= s.size() || s[i] != ':') fail("expected :");
      ++i;
      JVal val = value();
      v.obj.emplace_back(key, std::move(val));
      ws();
      if (i < s.size() && s[i] == ',') {
        ++i;
        continue;
      }
      if (i < s.size() && s[i] == '}') {
        ++i;
        return v;
      }
      fail("expected , or }");
    }
  }
};

const JVal* jfind(const JVal& o, const char* key) {
  for (auto& kv : o.obj)
    if (kv.first == key) return &kv.second;
  return nullptr;
}

float jfloat(const JVal& v, const char* key) {
  if (v.kind != JVal::Num) throw ParseError(std::string("type error for key ") + key);
  return static_cast<float>(v.num);  // JSON double, then narrowed to float
}

int jint(const JVal& v, const char* key) {
  if (v.kind != JVal::Num) throw ParseError(std::string("type error for key ") + key);
  return v.num_is_int ? static_cast<int>(v.inum) : static_cast<int>(v.num);
}

bool read_file(const std::string& path, std::string& text) {
  std::ifstream f(path, std::ios::binary);
  if (f.fail()) return false;
  std::stringstream ss;
  ss << f.rdbuf();
  text = ss.str();
  return true;
}

// ---------------------------------------------------------------------------
// Geometry, each function citing the reference routine it restates.

// RectangleReceiver::Cinit_vertex / setFocusCenter / Cset_resolution
// (Scene/DataStructure/Receiver/RectangleReceiver.cu:9-105).
void init_rectangle_receiver(ReceiverModel& r, int ppm) {
  r.pixel_length = 1.0f / float(ppm);
  switch (r.face) {
    case 0: r.local_normal = v3(0.0f, 0.0f, 1.0f); break;
    case 1: r.local_normal = v3(1.0f, 0.0f, 0.0f); break;
    case 2: r.local_normal = v3(0.0f, 0.0f, -1.0f); break;
    case 3: r.local_normal = v3(-1.0f, 0.0f, 0.0f); break;
    default: throw std::runtime_error("rectangle receiver face must be 0..3");
  }
  const float3 s = r.size;
  float3* v = r.vertex;
  switch (r.face) {
    case 0:
      v[0] = v3(-s.x / 2, -s.y / 2, s.z / 2);
      v[1] = v3(-s.x / 2, s.y / 2, s.z / 2);
      v[2] = v3(s.x / 2, s.y / 2, s.z / 2);
      v[3] = v3(s.x / 2, -s.y / 2, s.z / 2);
      break;
    case 1:
      v[0] = v3(s.x / 2, -s.y / 2, s.z / 2);
      v[1] = v3(s.x / 2, s.y / 2, s.z / 2);
      v[2] = v3(s.x / 2, s.y / 2, -s.z / 2);
      v[3] = v3(s.x / 2, -s.y / 2, -s.z / 2);
      break;
    case 2:
      v[0] = v3(s.x / 2, -s.y / 2, -s.z / 2);
      v[1] = v3(s.x / 2, s.y / 2, -s.z / 2);
      v[2] = v3(-s.x / 2, s.y / 2, -s.z / 2);
      v[3] = v3(-s.x / 2, -s.y / 2, -s.z / 2);
      break;
    default:
      v[0] = v3(-s.x / 2, -s.y / 2, -s.z / 2);
      v[1] = v3(-s.x / 2, s.y / 2, -s.z / 2);
      v[2] = v3(-s.x / 2, s.y / 2, s.z / 2);
      v[3] = v3(-s.x / 2, -s.y / 2, s.z / 2);
      break;
  }
  r.normal = normalize(r.normal);
  for (int k = 0; k < 4; ++k) v[k] = rotate_y(v[k], r.local_normal, r.normal);
  for (int k = 0; k < 4; ++k) v[k] = add(v[k], r.pos);
  r.focus = divs(add(v[0], v[2]), 2);
  r.resolution.x = int(r.size.x * float(ppm));
  r.resolution.y = int(r.size.y * float(ppm));
}

// CylinderReceiver::CInit / Cset_resolution (Scene/DataStructure/Receiver/CylinderReceiver.cu:4-15).
void init_cylinder_receiver(ReceiverModel& r, int ppm) {
  r.pixel_length = 1.0f / float(ppm);
  r.resolution.x = int(std::ceil(2 * M_PI * r.size.x * float(ppm)));
  r.resolution.y = int(r.size.y * float(ppm));
}

// CylinderReceiver::isInsideCylinder (CylinderReceiver.cuh:98-101).
bool inside_cylinder(const ReceiverModel& r, float3 p) {
  float2 l = make_float2(p.x - r.pos.x, p.z - r.pos.z);
  return dot2(l, l) <= r.size.x * r.size.x;
}

// Receiver::getFocusCenter for both receiver types
// (RectangleReceiver.cu:103-105; CylinderReceiver.cu:18-31).
float3 focus_center(const ReceiverModel& r, float3 helio_pos) {
  if (r.type == 0) return r.focus;
  if (inside_cylinder(r, helio_pos)) return r.pos;
  float3 dir = normalize(sub(helio_pos, r.pos));
  float radius = r.size.x / (length2(make_float2(dir.x, dir.z)));
  float x = r.pos.x + dir.x * radius;
  float z = r.pos.z + dir.z * radius;
  return v3(x, r.pos.y, z);
}

// Heliostat::CSetNormal and CSetWorldVertex (Scene/DataStructure/Heliostat/Heliostat.cu:15-40),
// with the focus-length reset of FocusFlatRectangleHelio::CSetNormalAndRotate
// (FocusFlatRectangleHelio.cu:333-339).
void orient_heliostat(HeliostatModel& h, float3 focus, float3 sun_dir) {
  if (h.type == 1 && h.focus_length < 0.0f) h.focus_length = length(sub(focus, h.pos));
  h.focus = focus;
  h.normal = helio_normal(h.pos, focus, sun_dir);
  flat_vertices(h.size, h.normal, h.pos, h.vertex);
}

// Sub-heliostat parallelograms of one heliostat, appended to `out`
// (RectangleHelio.cu:14-18; FocusFlatRectangleHelio.cu:123-227).
void sub_vertices(HeliostatModel& h, std::vector<float3>& out) {
  if (h.type == 0) {
    out.push_back(h.vertex[0]);
    out.push_back(h.vertex[1]);
    out.push_back(h.vertex[2]);
    return;
  }
  const int rows = h.row_col.x, cols = h.row_col.y;
  const float2 len = sub_lengths(h.size, h.gap, h.row_col);
  h.local_centers.assign(rows * cols, v3(0, 0, 0));
  h.local_normals.assign(rows * cols, v3(0, 0, 0));
  if (h.read_method == -1) {
    for (int r = 0; r < rows; ++r) {
      for (int c = 0; c < cols; ++c) {
        int id = r * cols + c;
        float3 cen = v3(c * (h.gap.x + len.y) - h.size.x / 2 + len.y / 2, h.size.y / 2,
                        r * (h.gap.y + len.x) - h.size.z / 2 + len.x / 2);
        cen.y += (cen.x * cen.x + cen.z * cen.z) / (4 * h.focus_length);
        h.local_centers[id] = cen;
        float3 nrm = v3(-1 / (2 * h.focus_length) * cen.x, 1.0f, -1 / (2 * h.focus_length) * cen.z);
        h.local_normals[id] = normalize(nrm);
      }
    }
  } else if (h.read_method == 1) {
    if ((int)h.file_local_centers.size() < rows * cols || (int)h.file_local_normals.size() < rows * cols)
      throw std::runtime_error("focus-flat heliostat reads its facets from the file but the subhelio block is short");
    for (int id = 0; id < rows * cols; ++id) {
      h.local_centers[id] = h.file_local_centers[id];
      h.local_normals[id] = normalize(h.file_local_normals[id]);
    }
  } else {
    throw std::runtime_error("focus-flat heliostat has no corresponding read method");
  }
  for (int id = 0; id < rows * cols; ++id) {
    float3 v[3];
    focus_flat_sub_vertices(len, h.local_centers[id], h.local_normals[id], h.normal, h.pos, v);
    out.insert(out.end(), v, v + 3);
  }
}

// RectangleGrid::CGridHelioMatch with boxIntersect
// (Scene/DataStructure/Grid/RectangleGrid.cu:27-117).  Builds the reference's
// sub-heliostat CSR and, over the same cells, a heliostat-level CSR.
void match_grid(GridModel& g, const std::vector<HeliostatModel>& hs) {
  const int3 n = g.cells;
  const long long ncell = (long long)n.x * n.y * n.z;
  if (ncell <= 0 || ncell > (1LL << 28)) throw std::runtime_error("grid cell count is out of range");
  std::vector<std::vector<int>> sub_lists(ncell), helio_lists(ncell);
  int start_sub = 0;
  for (int i = g.start_heliostat; i < g.start_heliostat + g.num_heliostats; ++i) {
    const HeliostatModel& h = hs[i];
    float radius = length(h.size) / 2;
    float3 lo = subs(h.pos, radius);
    float3 hi = adds(h.pos, radius);
    int3 lo_c = trunc3(cdiv(sub(lo, g.pos), g.interval));
    int3 hi_c = trunc3(cdiv(sub(hi, g.pos), g.interval));
    for (int x = std::max(0, lo_c.x); x <= std::min(n.x - 1, hi_c.x); ++x)
      for (int y = std::max(0, lo_c.y); y <= std::min(n.y - 1, hi_c.y); ++y)
        for (int z = std::max(0, lo_c.z); z <= std::min(n.z - 1, hi_c.z); ++z) {
          long long cell = (long long)x * n.y * n.z + (long long)y * n.z + z;
          for (int k = 0; k < h.num_sub; ++k) sub_lists[cell].push_back(start_sub + k);
          helio_lists[cell].push_back(i - g.start_heliostat);
        }
    start_sub += h.num_sub;
  }
  g.num_subheliostats = start_sub;
  g.cell_index.assign(ncell + 1, 0);
  g.cell_hindex.assign(ncell + 1, 0);
  g.cell_match.clear();
  g.cell_hmatch.clear();
  for (long long c = 0; c < ncell; ++c) {
    g.cell_index[c + 1] = g.cell_index[c] + (int)sub_lists[c].size();
    g.cell_hindex[c + 1] = g.cell_hindex[c] + (int)helio_lists[c].size();
    g.cell_match.insert(g.cell_match.end(), sub_lists[c].begin(), sub_lists[c].end());
    g.cell_hmatch.insert(g.cell_hmatch.end(), helio_lists[c].begin(), helio_lists[c].end());
  }
}

}  // namespace

// ---------------------------------------------------------------------------
void facet_lattice(const HeliostatModel& h, float pixel_length, int2& sub_row_col, float2& sub_length,
                   int& num_facets) {
  sub_length.x = (h.size.z - h.gap.y * (h.row_col.x - 1)) / float(h.row_col.x);
  sub_length.y = (h.size.x - h.gap.x * (h.row_col.y - 1)) / float(h.row_col.y);
  sub_row_col.x = int(sub_length.x / pixel_length);
  sub_row_col.y = int(sub_length.y / pixel_length);
  long long n = (long long)h.row_col.x * h.row_col.y * sub_row_col.x * sub_row_col.y;
  if (n < 0 || n > 0x7fffffffLL) throw std::runtime_error("heliostat micro-facet count overflows int");
  num_facets = (int)n;
}

bool read_scene_text(const std::string& text, SceneModel& scene, std::string& err) {
  int2 matrix = make_int2(1, 1);
  float2 gap = make_float2(0.0f, 0.0f);
  float surface[6] = {-1, -1, -1, -1, -1, -1};
  std::vector<float3> centers, normals;
  std::string head;
  int receiver_id = -1, grid_id_for_receiver = 0, helio_id_for_grid = 0, total_helios = 0;
  int n_centers = 0, n_normals = 0, n_sub = 0;
  int helio_type = -1;
  St state = St::Start;
  scene = SceneModel();
  std::istringstream in(text);
  try {
    while (in >> head) {
      if (head[0] == '#') {
        std::string rest;
        std::getline(in, rest);
        continue;
      }
      if (head == "gap") {
        in >> gap.x >> gap.y;
      } else if (head == "matrix") {
        in >> matrix.x >> matrix.y;
      } else if (head == "surface_property") {
        for (int k = 0; k < 6; ++k) in >> surface[k];
      } else if (head == "ground") {
        state = step(state, 'D');
        in >> scene.ground_length >> scene.ground_width;
        scene.grid_num = int_field(in, "ngrid");
      } else if (head == "Recv") {
        state = step(state, 'R');
        int type = -1;
        in >> type;
        if (type != 0 && type != 1) throw std::runtime_error("Receiver type has not defined.\n");
        ReceiverModel r;
        r.type = type;
        r.pos = float3_field(in, "pos");
        r.size = float3_field(in, "size");
        r.normal = float3_field(in, "norm");
        r.face = int_field(in, "face");
        expect_key(in, "end");
        scene.receivers.push_back(r);
        ++receiver_id;
        grid_id_for_receiver = 0;
      } else if (head == "Grid") {
        state = step(state, 'G');
        int type = -1;
        in >> type;
        if (type != 0) throw std::runtime_error("Grid type has not defined.\n");
        GridModel g;
        g.type = type;
        g.receiver = receiver_id;
        g.start_heliostat = total_helios;
        g.pos = float3_field(in, "pos");
        g.size = float3_field(in, "size");
        g.interval = float3_field(in, "inter");
        g.num_heliostats = int_field(in, "n");
        g.heliostat_type = int_field(in, "type");
        expect_key(in, "end");
        scene.grids.push_back(g);
        helio_type = g.heliostat_type;
        ++grid_id_for_receiver;
        helio_id_for_grid = 0;
      } else if (head == "helio") {
        state = step(state, 'H');
        if (helio_type != 0 && helio_type != 1) throw std::runtime_error("Heliostat has not defined.\n");
        HeliostatModel h;
        h.type = helio_type;
        if (int(surface[1]) == 1) {
          h.file_local_centers = centers;
          h.file_local_normals = normals;
        }
        h.gap = gap;
        h.row_col = matrix;
        for (int k = 0; k < 6; ++k) h.surface_property[k] = surface[k];
        if (h.type == 1) {
          h.focus_length = surface[0];
          h.read_method = int(surface[1]);
        }
        in >> h.pos.x >> h.pos.y >> h.pos.z;
        in >> h.size.x >> h.size.y >> h.size.z;
        h.grid = (int)scene.grids.size() - 1;
        scene.heliostats.push_back(h);
        n_sub = n_normals = n_centers = 0;
        centers.clear();
        normals.clear();
        ++helio_id_for_grid;
        ++total_helios;
      } else if (head == "subhelio") {
        std::string rest;
        std::getline(in, rest);
        for (; n_centers < matrix.x * matrix.y; ++n_centers) {
          float a, b, c;
          in >> a >> b >> c;
          centers.push_back(v3(a, b, c));
          std::getline(in, rest);
          ++n_sub;
        }
        for (; n_normals < matrix.x * matrix.y; ++n_normals) {
          float a, b, c;
          in >> a >> b >> c;
          normals.push_back(v3(a, b, c));
          std::getline(in, rest);
          ++n_sub;
        }
      } else {
        state = step(state, '?');
      }
    }
    // SceneLoader::checkScene (Scene/SceneLoader.cpp:200-238).
    if (scene.grid_num != (int)scene.grids.size())
      throw ParseError("The scene should contains " + std::to_string(scene.grid_num) + " grids, but got " +
                       std::to_string(scene.grids.size()) + " grids.");
    for (size_t i = 0; i < scene.grids.size(); ++i) {
      int expect = scene.grids[i].num_heliostats;
      int exist = (i + 1 == scene.grids.size()) ? (int)scene.heliostats.size() : scene.grids[i + 1].start_heliostat;
      exist -= scene.grids[i].start_heliostat;
      if (exist != expect)
        throw ParseError("The " + std::to_string(i + 1) + "-th grid should contain " + std::to_string(expect) +
                         " heliostat(s), but got " + std::to_string(exist) + " heliostat(s).");
      int recv = scene.grids[i].receiver;
      if (i == 0 && recv != 0) throw ParseError("The 0-th grid is expected belonging to 0-th receiver.");
      if (i > 0) {
        int prev = scene.grids[i - 1].receiver;
        if (recv != prev && recv != prev + 1)
          throw ParseError("The " + std::to_string(i) + "-th grid has a receiver index out of order.");
      }
    }
    return true;
  } catch (const ParseError& e) {
    err = std::string("Error caused by ' ") + e.what() + " '.";
    return false;
  } catch (const std::exception& e) {
    err = "Error occurs at " + std::to_string(receiver_id + 1) + "-th receiver, " +
          std::to_string(grid_id_for_receiver) + "-th grid, " + std::to_string(helio_id_for_grid) +
          "-th heliostat with head '" + head + "'. This is caused by ' " + e.what() + "'";
    return false;
  }
}

bool read_scene_file(const std::string& path, SceneModel& scene, std::string& err) {
  std::string text;
  if (!read_file(path, text)) {
    err = "Cannot open the file: " + path;
    scene = SceneModel();
    return false;
  }
  return read_scene_text(text, scene, err);
}

int read_config_text(const std::string& text, SceneConfig& c, std::string& err) {
  try {
    JParser p(text);
    JVal root = p.value();
    p.ws();
    if (p.i != text.size()) p.fail("trailing characters");
    if (root.kind != JVal::Obj) throw ParseError("configuration must be a JSON object");
    int n = 0;
    if (const JVal* v = jfind(root, "sun_dir")) {
      if (v->kind != JVal::Arr || v->arr.size() < 3) throw ParseError("sun_dir must be an array of 3 numbers");
      c.sun_dir.x = jfloat(v->arr[0], "sun_dir");
      c.sun_dir.y = jfloat(v->arr[1], "sun_dir");
      c.sun_dir.z = jfloat(v->arr[2], "sun_dir");
      ++n;
    }
    if (const JVal* v = jfind(root, "dni")) c.dni = jfloat(*v, "dni"), ++n;
    if (const JVal* v = jfind(root, "csr")) c.csr = jfloat(*v, "csr"), ++n;
    if (const JVal* v = jfind(root, "num_of_sunshape_groups")) c.num_sunshape_groups = jint(*v, "num_of_sunshape_groups"), ++n;
    if (const JVal* v = jfind(root, "num_per_sunshape_group")) c.num_per_sunshape_group = jint(*v, "num_per_sunshape_group"), ++n;
    if (const JVal* v = jfind(root, "inverse_transform_sampling_groups"))
      c.inverse_transform_sampling_groups = jint(*v, "inverse_transform_sampling_groups"), ++n;
    if (const JVal* v = jfind(root, "receiver_pixel_length")) c.receiver_pixel_length = jfloat(*v, "receiver_pixel_length"), ++n;
    if (const JVal* v = jfind(root, "helio_disturb_std")) c.helio_disturb_std = jfloat(*v, "helio_disturb_std"), ++n;
    if (const JVal* v = jfind(root, "helio_pixel_length")) c.helio_pixel_length = jfloat(*v, "helio_pixel_length"), ++n;
    if (const JVal* v = jfind(root, "helio_reflected_rate")) c.helio_reflected_rate = jfloat(*v, "helio_reflected_rate"), ++n;
    return n;
  } catch (const std::exception& e) {
    err = e.what();
    return -1;
  }
}

int read_config_file(const std::string& path, SceneConfig& c, std::string& err) {
  std::string text;
  if (!read_file(path, text)) {
    err = "The file '" + path + "' doesn't exist";
    return -1;
  }
  return read_config_text(text, c, err);
}

bool process_scene(SceneModel& s, std::string& err) {
  try {
    if (s.receivers.empty() || s.grids.empty()) throw std::runtime_error("scene has no receiver or grid");
    const SceneConfig& cfg = s.config;
    if (!(cfg.receiver_pixel_length > 0.0f) || !(cfg.helio_pixel_length > 0.0f))
      throw std::runtime_error("pixel lengths must be positive");
    const int ppm = int(1.0f / cfg.receiver_pixel_length);
    if (ppm <= 0) throw std::runtime_error("receiver pixel length is larger than one metre");
    for (auto& h : s.heliostats) {
      h.num_sub = (h.type == 1) ? h.row_col.x * h.row_col.y : 1;
      if (h.row_col.x <= 0 || h.row_col.y <= 0) throw std::runtime_error("heliostat matrix must be positive");
    }
    for (auto& g : s.grids) {
      if (g.receiver < 0 || g.receiver >= (int)s.receivers.size()) throw std::runtime_error("grid receiver index is invalid");
      g.cells.x = int(std::ceil(g.size.x / g.interval.x));
      g.cells.y = int(std::ceil(g.size.y / g.interval.y));
      g.cells.z = int(std::ceil(g.size.z / g.interval.z));
      match_grid(g, s.heliostats);
      ReceiverModel& r = s.receivers[g.receiver];
      if (r.type == 0)
        init_rectangle_receiver(r, ppm);
      else
        init_cylinder_receiver(r, ppm);
      if (r.resolution.x <= 0 || r.resolution.y <= 0) throw std::runtime_error("receiver resolution is empty");
      for (int i = 0; i < g.num_heliostats; ++i) {
        HeliostatModel& h = s.heliostats[g.start_heliostat + i];
        float3 focus = focus_center(r, h.pos);
        h.pixel_length = cfg.helio_pixel_length;
        orient_heliostat(h, focus, cfg.sun_dir);
      }
    }
    for (auto& g : s.grids) {
      g.sub_vertices.clear();
      int sub = 0;
      for (int i = 0; i < g.num_heliostats; ++i) {
        HeliostatModel& h = s.heliostats[g.start_heliostat + i];
        h.sub_begin = sub;
        sub += h.num_sub;
        sub_vertices(h, g.sub_vertices);
        facet_lattice(h, h.pixel_length, h.sub_row_col, h.sub_length, h.num_facets);
      }
    }
    s.processed = true;
    return true;
  } catch (const std::exception& e) {
    err = e.what();
    return false;
  }
}

void set_sun(SceneModel& s, float3 sun_dir) {
  s.config.sun_dir = sun_dir;
  for (auto& h : s.heliostats) orient_heliostat(h, h.focus, sun_dir);
  for (auto& g : s.grids) {
    g.sub_vertices.clear();
    for (int i = 0; i < g.num_heliostats; ++i) sub_vertices(s.heliostats[g.start_heliostat + i], g.sub_vertices);
  }
}

int read_task_file(const std::string& path, const SceneModel& scene, std::vector<int>& heliostats,
                   std::vector<int>& receivers, std::string& err) {
  heliostats.clear();
  receivers.clear();
  std::ifstream f(path);
  if (f.fail()) {
    err = "Cannot open the file '" + path + "'.";
    return -1;
  }
  std::stringstream in;
  in << f.rdbuf();
  f.close();
  std::string tok;
  in >> tok;
  int n = 0;
  size_t used = 0;
  try {
    n = std::stoi(tok, &used);
  } catch (...) {
    err = "The number of heliostats '" + tok + "' is invalid.";
    return -1;
  }
  if (used < tok.size() || n <= 0) {
    err = "The number of heliostats '" + tok + "' is invalid.";
    return -1;
  }
  int ans = 1;
  for (int i = 0; i < n; ++i) {
    if (in.rdbuf()->in_avail() == 0) {
      err = std::to_string(n) + " heliostat(s) are expected. But only got " + std::to_string(i) + " heliostats.";
      return -1;
    }
    in >> tok;
    int id = 0;
    try {
      id = std::stoi(tok, &used);
    } catch (...) {
      err = "The " + std::to_string(i + 1) + "-th heliostat index '" + tok + "' is invalid.";
      return -1;
    }
    if (used < tok.size() || id < 0 || id >= (int)scene.heliostats.size()) {
      err = "The " + std::to_string(i + 1) + "-th heliostat index '" + tok + "' is invalid.";
      return -1;
    }
    if (std::find(heliostats.begin(), heliostats.end(), id) == heliostats.end()) {
      heliostats.push_back(id);
      int grid = scene.heliostats[id].grid;
      if (std::find(receivers.begin(), receivers.end(), grid) == receivers.end()) receivers.push_back(grid);
    } else {
      ans = 0;
    }
  }
  std::string rest;
  in >> rest;
  if (!rest.empty()) return 0;
  return ans;
}

float save_text_image(const std::string& path, int height, int width, const float* data, int precision,
                      std::string& err, bool* ok) {
  FILE* fp = std::fopen(path.c_str(), "w");
  if (!fp) {
    err = "cannot open '" + path + "' for writing";
    if (ok) *ok = false;
    return 0.0f;
  }
  float max_value = 0.0f;
  std::string line;
  char buf[64];
  for (int r = 0; r < height; ++r) {
    line.clear();
    const float* row = data + (size_t)(height - 1 - r) * width;
    for (int c = 0; c < width; ++c) {
      float v = row[c];
      if ((double)v < kEps) {
        line.push_back('0');
      } else {
        max_value = std::max(max_value, v);
        std::snprintf(buf, sizeof(buf), "%.*f", precision, (double)v);
        line.append(buf);
      }
      line.push_back(c != width - 1 ? ',' : '\n');
    }
    std::fwrite(line.data(), 1, line.size(), fp);
  }
  std::fclose(fp);
  if (ok) *ok = true;
  return max_value;
}

}  // namespace qm
