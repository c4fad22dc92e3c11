// The engine's host side: the design records, the placer's construction and the initial
// placement's host half (B2B assembly), restating vyges-gpl's Rust function by function (each
// cites its file:line). The construction is integer work and stays on the CPU; the solves and
// the Nesterov loop run on the device (engine.h).
#pragma once
#include <array>
#include <functional>
#include <cmath>
#include <cstdint>
#include <tuple>
#include <map>
#include <string>
#include <vector>

#include "../../../include/gpl.h"

namespace gpl {

// ---- Rust `as` conversions: saturating, NaN to 0 ----
inline int32_t f2i(double v) {
  if (std::isnan(v)) return 0;
  if (v >= 2147483647.0) return INT32_MAX;
  if (v <= -2147483648.0) return INT32_MIN;
  return (int32_t)v;
}
inline int64_t f2l(double v) {
  if (std::isnan(v)) return 0;
  if (v >= 9223372036854775807.0) return INT64_MAX;
  if (v <= -9223372036854775808.0) return INT64_MIN;
  return (int64_t)v;
}
inline uint64_t f2ul(double v) {
  if (std::isnan(v) || v <= 0) return 0;
  if (v >= 18446744073709551615.0) return UINT64_MAX;
  return (uint64_t)v;
}
// f32::max / f32::min (IEEE maxNum: a NaN operand yields the other)
inline float fmaxr(float a, float b) { return std::fmax(a, b); }
inline float fminr(float a, float b) { return std::fmin(a, b); }

// ---- how a run stops (src/log.rs:18-28) ----
struct StopEx {
  bool error;            // true: the reference's error (its line printed); false: refused
  std::string tool;
  int id = 0;
  std::string why;
};
[[noreturn]] void refuse(const std::string &why);

// ---- the logger (src/log.rs:9-107): "[INFO GPL-0001] msg", a 1000-per-code limit ----
struct Log {
  std::vector<std::string> lines;
  std::vector<std::string> trace;
  std::map<std::string, int> counts;
  bool trace_on = false;
  void emit(const char *level, const std::string &tool, int id, const std::string &msg);
  void info(const std::string &tool, int id, const std::string &msg) { emit("INFO", tool, id, msg); }
  void warn(const std::string &tool, int id, const std::string &msg) { emit("WARNING", tool, id, msg); }
  [[noreturn]] void error(const std::string &tool, int id, const std::string &msg);
  void report(const std::string &msg);
  void probe(const std::string &line) {
    if (trace_on) trace.push_back(line);
  }
};

std::string sfmt(const char *f, ...) __attribute__((format(printf, 1, 2)));
// Rust `{}` Display of a float: shortest round-trip digits, never an exponent.
std::string rust_f32(float v);
std::string rust_f64(double v);
// fmt_e (src/nesterov.rs:2086-2092), fmt_g (:2114-2135), fmt_g_prec (:2097-2112).
std::string fmt_e(double v, int prec, int width);
std::string fmt_g(double v);
std::string fmt_g_prec(double v, int p);
// log.rs fmt_f32 / fmt_f64 / fmt_e (src/log.rs:114-149).
std::string log_fmt_f32(float v);
std::string log_fmt_f64(double v);
std::string log_fmt_e(double v, int digits);

// ---- the design records (src/placer_base.rs:17-206) ----
struct Rect {
  int32_t lx = 0, ly = 0, ux = 0, uy = 0;
  int32_t dx() const { return ux - lx; }
  int32_t dy() const { return uy - ly; }
  int64_t area() const { return (int64_t)dx() * (int64_t)dy(); }
  Rect intersect(const Rect &o) const;
  bool contains(const Rect &o) const { return lx <= o.lx && ly <= o.ly && o.ux <= ux && o.uy <= uy; }
};

struct DbInst {
  std::string name, master;
  bool core_auto_placeable = true, master_is_block = false, fixed = false, placed = false;
  Rect bbox;
  int group = -1;
  bool has_halo = false;
  Rect halo;
  int64_t signal_pins = 0;
  int orient = GPL_R0;
  int32_t master_w = 0, master_h = 0;
};
struct Term {
  int inst = 0;
  bool has_shape = false;
  Rect shape;
  int order = 0;
};
struct Port {
  std::string name;
  bool has_bbox = false;
  Rect bbox;
  bool fixed = false;
};
struct DbNet {
  std::string name;
  bool signal_or_clock = true;
  std::vector<Term> iterms;
  std::vector<Port> bterms;
};
struct Group {
  std::string name;
  bool visual_debug = false;
  int region = -1;
};
struct Region {
  std::vector<Rect> boundaries;
  std::vector<int> groups;
};
struct Blockage {
  Rect bbox;
  int inst = -1;
  bool inst_fixed = false;
  std::string inst_name;
  float max_density = 0;
};
struct RowRec {
  Rect box;
  bool pad = false;
  int32_t site_w = 0, site_h = 0;
};
struct Design {
  int32_t dbu = 1000;
  Rect die, core;
  std::vector<RowRec> rows;
  std::vector<DbInst> insts;
  std::vector<DbNet> nets;
  std::vector<Group> groups;
  std::vector<Region> regions;
  std::vector<Blockage> blockages;
};
Design design_from_c(const gpl_design_t *c);

// ---- the placer (src/placer_base.rs:208-491) ----
struct Vars {
  int32_t pad_left = 0, pad_right = 0;
  bool skip_io = false, place_ios = false, disable_pin_density_adjust = false;
};
struct Instance {
  int db = -1;  // design instance, -1 for a dummy
  int32_t lx = 0, ly = 0, ux = 0, uy = 0;
  bool fixed = false, macro_ = false, locked = false;
  int32_t dx() const { return ux - lx; }
  int32_t dy() const { return uy - ly; }
  int32_t cx() const { return (lx + ux) / 2; }
  int32_t cy() const { return (ly + uy) / 2; }
  int64_t area() const { return (int64_t)dx() * (int64_t)dy(); }
  bool is_place_instance() const { return db >= 0 && !fixed; }
  int64_t extend_size_by_scale(double scale);
  void snap_outward(int32_t ox, int32_t oy, int32_t sx, int32_t sy);
};
struct Common {
  int32_t site_x = 0, site_y = 0;
  std::vector<Instance> insts;
  std::vector<std::pair<int, int64_t>> nets;  // (design net, pin count)
  int64_t pins = 0;
};
struct Base {
  int group = -1;
  Rect region_bbox;
  int64_t region_area = 0;
  std::vector<int> place_insts, fixed_insts;
  std::vector<Instance> dummies;
  int64_t place_insts_area = 0, non_place_insts_area = 0, std_insts_area = 0, macro_insts_area = 0;
};
std::pair<int32_t, int32_t> min_max_idx(int32_t ll, int32_t uu, int32_t core_ll, int32_t site, int32_t mn, int32_t mx);
Common placer_base_common(Log &log, const Design &d, const Vars &v);
Base placer_base(Log &log, const Design &d, const Common &c, int group, bool check_density);

// ---- initial placement (src/initial_place.rs, src/bicgstab.rs) ----
struct IpVars {
  int max_iter = 20;
  int32_t min_diff_length = 1500;
  int max_solver_iter = 100;
  int max_fanout = 200;
  float net_weight_scale = 800.0f;
  bool force_center = false;
};
struct Pin {
  int inst = -1;  // placer instance
  bool port = false, movable_io = false;
  int32_t off_x = 0, off_y = 0, cx = 0, cy = 0;
  bool min_x = false, max_x = false, min_y = false, max_y = false;
};
// Lists of pin indices, one per owner (a net, an instance), stored flat: owner k's pins are
// items[start[k] .. start[k + 1]). The reference keeps a vector per owner; one array of all
// of them builds without a heap block per owner.
struct PinLists {
  struct Span {
    const int *b = nullptr, *e = nullptr;
    const int *begin() const { return b; }
    const int *end() const { return e; }
    size_t size() const { return (size_t)(e - b); }
    bool empty() const { return b == e; }
    int operator[](size_t i) const { return b[i]; }
  };
  std::vector<int64_t> start{0};
  std::vector<int> items;
  size_t size() const { return start.size() - 1; }
  Span operator[](size_t k) const { return {items.data() + start[k], items.data() + start[k + 1]}; }
  int *begin_of(size_t k) { return items.data() + start[k]; }
  int *end_of(size_t k) { return items.data() + start[k + 1]; }
};

struct Ip {
  std::vector<Pin> pins;
  PinLists net_pins;
  std::vector<Rect> db_bbox;
  std::vector<int> place;
  PinLists inst_pins;
};

// ---- random numbers (src/normal.rs) ----
struct Mt19937 {
  uint32_t x[624];
  int i = 624;
  explicit Mt19937(uint32_t seed);
  uint32_t next_u32();
  void twist();
};
int32_t uniform_int(Mt19937 &eng, int32_t mn, int32_t mx);
double normal(Mt19937 &eng, double mean, double sigma);

std::pair<int32_t, int32_t> orient_point(int orient, int32_t x, int32_t y);
Ip make_pins(const Design &d, const Common &c, const Vars &v);
class IpDevice;
Ip do_bicgstab_place_device(Log &log, const Design &d, Common &c, const Vars &v, const IpVars &vars, IpDevice &dev);

}  // namespace gpl

namespace gpl {
// Progress lines on stderr, with the seconds since the first call, when GPL_LOG is set in the
// environment (timings of the host phases; the run's report is unaffected).
void progress(const char *fmt, ...) __attribute__((format(printf, 1, 2)));
}  // namespace gpl
