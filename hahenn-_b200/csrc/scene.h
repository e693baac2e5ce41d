// Scene JSON → tank geometry, obstacles, drains, water blocks and sources.
//
// Accepts the reference's scene file ({v:1, app:'suiri-lab', scene:{tank:{w,h,d}, items:[…]}, cam},
// src/js/80-ui.js:121) or a bare {tank, items}. Every item field is checked against the defaults of a
// fresh item of the same kind and falls back to them, as the reference's validScene does
// (src/js/80-ui.js:430-459); items are in solver coordinates (y up).
#pragma once
#include <string>
#include <utility>
#include <vector>

#include "common.cuh"

namespace suiri {

struct JVal {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  double num = 0.0;
  bool b = false;
  std::string s;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
  const JVal* get(const char* key) const;
  bool is_num() const { return kind == Num; }
};

bool json_parse(const std::string& text, JVal& out, std::string& err);

struct WaterBlock { double lo[3], hi[3]; };

struct SourceItem {
  int id = 0;
  std::string mode = "stream";
  bool enabled = true;
  double pos[3] = {0, 0.4, 0};
  double pitch = -90, yaw = 0;
  double flow = 3.0, speed = 0.6, drop_d = 5, drop_rate = 3, spread = 18, burst = 0.5, burst_every = 0;
  double rain_rate = 60, rain_size = 0.3, total = 0;
};

struct SceneItem {             // an obstacle or drain as given (for velocities from the previous transform)
  int id = 0;
  Obj obj{};
  double R[9];                 // world-from-local rotation
};

struct Scene {
  double tank[3] = {0.6, 0.32, 0.4};     // w, h (up), d
  std::vector<SceneItem> solids;          // obstacles (flag 1) and drains (flag 2)
  std::vector<WaterBlock> blocks;
  std::vector<SourceItem> sources;
  std::string items_json;                 // the validated items as JSON (every field filled, ids assigned)
};

// items only (for set_objects); returns false with err on malformed JSON
bool parse_items(const JVal& items, Scene& sc, std::string& err);
// a whole scene file; clamp_tank applies the editor's tank limits (w∈[0.2,1.2], h∈[0.1,0.6], d∈[0.15,1])
bool parse_scene(const std::string& text, bool clamp_tank, Scene& sc, std::string& err);

// the validated scene {tank, items} as JSON text (what the reference's validScene returns)
std::string scene_json_text(const Scene& sc);

void euler_deg(double rx, double ry, double rz, double R[9]);
// (type, d0..d3) of an obstacle shape (src/js/10-scene.js:143-157); false for an unknown shape
bool shape_params(const std::string& shape, const JVal* dims, int& type, double d[4]);
double bound_radius(int type, const double d[4]);

}  // namespace suiri
