// Oracle, part 1: the logger and its formats, the design records, the placer's construction
// (src/placer_base.rs), the initial placement (src/initial_place.rs) and its solver
// (src/bicgstab.rs), and the random numbers (src/normal.rs). Test infrastructure only.
#include <algorithm>
#include <charconv>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <numeric>
#include <tuple>

#include "oracle.h"

namespace orc {

#include "../gpl_b200/csrc/host/ziggurat_tables.inc"

void refuse(const std::string &why) { throw StopEx{false, "", 0, why}; }

std::string sfmt(const char *f, ...) {
  char buf[4096];
  va_list ap;
  va_start(ap, f);
  int n = vsnprintf(buf, sizeof buf, f, ap);
  va_end(ap);
  if (n < (int)sizeof buf) return std::string(buf, n);
  std::string s(n + 1, '\0');
  va_start(ap, f);
  vsnprintf(&s[0], n + 1, f, ap);
  va_end(ap);
  s.resize(n);
  return s;
}

// The suite logger's line format (src/log.rs:151-197): a coded line "[LEVEL TOOL-NNNN] text",
// a message with newlines split into lines (the continuation lines bare), and at most 1000
// prints per code, the 1001st replaced by the limit notice.
void Log::emit(const char *level, const std::string &tool, int id, const std::string &msg) {
  std::string code = sfmt("%s-%04d", tool.c_str(), id);
  int &n = counts[code];
  n++;
  if (n > 1001) return;
  if (n == 1001) {
    lines.push_back(sfmt("[%s %s] message limit (1000) reached. This message will no longer print.", level, code.c_str()));
    return;
  }
  size_t start = 0;
  bool first = true;
  while (true) {
    size_t nl = msg.find('\n', start);
    std::string part = msg.substr(start, nl == std::string::npos ? std::string::npos : nl - start);
    if (first)
      lines.push_back(sfmt("[%s %s] %s", level, code.c_str(), part.c_str()));
    else
      lines.push_back(part);
    first = false;
    if (nl == std::string::npos) break;
    start = nl + 1;
  }
}
void Log::error(const std::string &tool, int id, const std::string &msg) {
  emit("ERROR", tool, id, msg);
  throw StopEx{true, tool, id, ""};
}
void Log::report(const std::string &msg) {
  size_t start = 0;
  while (true) {
    size_t nl = msg.find('\n', start);
    lines.push_back(msg.substr(start, nl == std::string::npos ? std::string::npos : nl - start));
    if (nl == std::string::npos) break;
    start = nl + 1;
  }
}

// Shortest round-trip digits of v (scientific), split into digit string and decimal exponent.
template <class F>
static void shortest(F v, std::string &digits, int &exp10, bool &neg) {
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof buf, v, std::chars_format::scientific);
  std::string s(buf, r.ptr);
  neg = s[0] == '-';
  if (neg) s = s.substr(1);
  size_t e = s.find('e');
  std::string m = s.substr(0, e);
  exp10 = std::atoi(s.c_str() + e + 1);
  digits.clear();
  for (char ch : m)
    if (ch != '.') digits.push_back(ch);
}

template <class F>
static std::string rust_display(F v) {
  if (std::isnan(v)) return "NaN";
  if (std::isinf(v)) return v < 0 ? "-inf" : "inf";
  if (v == 0) return std::signbit(v) ? "-0" : "0";
  std::string dg;
  int e;
  bool neg;
  shortest(v, dg, e, neg);
  std::string out;
  int n = (int)dg.size();
  if (e >= 0) {
    if (e + 1 >= n) {
      out = dg + std::string(e + 1 - n, '0');
    } else {
      out = dg.substr(0, e + 1) + "." + dg.substr(e + 1);
    }
  } else {
    out = "0." + std::string(-e - 1, '0') + dg;
  }
  return (neg ? "-" : "") + out;
}
std::string rust_f32(float v) { return rust_display(v); }
std::string rust_f64(double v) { return rust_display(v); }

template <class F>
static std::string rust_exp(F v) {  // Rust `{:e}`: shortest digits, "1.5e-14"
  std::string dg;
  int e;
  bool neg;
  shortest(v, dg, e, neg);
  std::string m = dg.substr(0, 1);
  if (dg.size() > 1) m += "." + dg.substr(1);
  return (neg ? "-" : "") + m + "e" + std::to_string(e);
}

template <class F>
static std::string log_fmt_g(F v) {
  bool finite_nonzero = std::isfinite(v) && v != 0;
  std::string fixed = rust_display(v);
  if (!finite_nonzero) {
    if (fixed == "NaN") return "nan";
    if (fixed == "inf" || fixed == "-inf") return fixed;
    return fixed;
  }
  std::string sci = rust_exp(v);
  size_t e = sci.find('e');
  std::string mant = sci.substr(0, e);
  int exp = std::atoi(sci.c_str() + e + 1);
  if (exp >= -4 && exp < 16) return fixed;
  return sfmt("%se%c%02d", mant.c_str(), exp < 0 ? '-' : '+', std::abs(exp));
}
std::string log_fmt_f32(float v) { return log_fmt_g(v); }
std::string log_fmt_f64(double v) { return log_fmt_g(v); }
std::string log_fmt_e(double v, int digits) { return sfmt("%.*e", digits, v); }

// fmt's `{:W.Pe}`: C's %e already writes a signed exponent of at least two digits.
std::string fmt_e(double v, int prec, int width) { return sfmt("%*.*e", width, prec, v); }

static std::string strip_zeros(const std::string &s) {
  if (s.find('.') == std::string::npos) return s;
  std::string t = s;
  while (!t.empty() && t.back() == '0') t.pop_back();
  if (!t.empty() && t.back() == '.') t.pop_back();
  return t;
}
std::string fmt_g_prec(double v, int p) {
  if (v == 0.0) return "0";
  p = std::max(p, 1);
  std::string e_form = sfmt("%.*e", p - 1, v);
  size_t e = e_form.find('e');
  std::string m = e_form.substr(0, e);
  int x = std::atoi(e_form.c_str() + e + 1);
  if (x < -4 || x >= p) return sfmt("%se%c%02d", strip_zeros(m).c_str(), x < 0 ? '-' : '+', std::abs(x));
  int decimals = std::max(p - 1 - x, 0);
  return strip_zeros(sfmt("%.*f", decimals, v));
}
std::string fmt_g(double v) {
  if (v == 0.0) return "0";
  int exp = (int)std::floor(std::log10(std::fabs(v)));
  if (!(exp >= -4 && exp < 6)) {
    std::string s = sfmt("%.5e", v);
    size_t e = s.find('e');
    std::string m = s.substr(0, e);
    int ee = std::atoi(s.c_str() + e + 1);
    return sfmt("%se%c%02d", strip_zeros(m).c_str(), ee < 0 ? '-' : '+', std::abs(ee));
  }
  int decimals = std::max(5 - exp, 0);
  return strip_zeros(sfmt("%.*f", decimals, v));
}

Rect Rect::intersect(const Rect &o) const {
  Rect r{std::max(lx, o.lx), std::max(ly, o.ly), std::min(ux, o.ux), std::min(uy, o.uy)};
  if (r.lx > r.ux || r.ly > r.uy) return Rect{};
  return r;
}

static Rect rect4(const int32_t *p) { return Rect{p[0], p[1], p[2], p[3]}; }

Design design_from_c(const gpl_design_t *c) {
  Design d;
  d.dbu = c->dbu;
  d.die = rect4(c->die);
  d.core = rect4(c->core);
  for (int r = 0; r < c->n_rows; r++) d.rows.push_back(RowRec{rect4(c->row_box + 4 * r), c->row_pad[r] != 0, c->row_site[2 * r], c->row_site[2 * r + 1]});
  d.insts.resize(c->n_insts);
  for (int k = 0; k < c->n_insts; k++) {
    DbInst &i = d.insts[k];
    i.name = c->inst_name ? c->inst_name[k] : sfmt("i%d", k);
    i.master = c->inst_master_name ? c->inst_master_name[k] : sfmt("m%d", k);
    uint32_t f = c->inst_flags[k];
    i.core_auto_placeable = f & GPL_INST_CORE_AUTO_PLACEABLE;
    i.master_is_block = f & GPL_INST_BLOCK;
    i.fixed = f & GPL_INST_FIXED;
    i.placed = f & GPL_INST_PLACED;
    i.bbox = rect4(c->inst_box + 4 * k);
    i.group = c->inst_group ? c->inst_group[k] : -1;
    i.has_halo = (f & GPL_INST_HAS_HALO) && c->inst_halo;
    if (i.has_halo) i.halo = rect4(c->inst_halo + 4 * k);
    i.signal_pins = c->inst_signal_pins[k];
    i.orient = c->inst_orient ? c->inst_orient[k] : GPL_R0;
    i.master_w = c->inst_master[2 * k];
    i.master_h = c->inst_master[2 * k + 1];
  }
  d.nets.resize(c->n_nets);
  for (int n = 0; n < c->n_nets; n++) {
    DbNet &net = d.nets[n];
    net.name = c->net_name ? c->net_name[n] : sfmt("n%d", n);
    net.signal_or_clock = c->net_signal[n] != 0;
    for (int64_t t = c->net_iterm_start[n]; t < c->net_iterm_start[n + 1]; t++) {
      Term tm;
      tm.inst = c->iterm_inst[t];
      tm.has_shape = c->iterm_has_shape[t] != 0;
      tm.shape = rect4(c->iterm_shape + 4 * t);
      tm.order = c->iterm_order[t];
      net.iterms.push_back(tm);
    }
    for (int64_t t = c->net_bterm_start[n]; t < c->net_bterm_start[n + 1]; t++) {
      Port p;
      p.name = c->bterm_name ? c->bterm_name[t] : sfmt("p%ld", (long)t);
      p.has_bbox = c->bterm_flags[t] & GPL_BTERM_PLACED;
      p.bbox = rect4(c->bterm_box + 4 * t);
      p.fixed = c->bterm_flags[t] & GPL_BTERM_FIXED;
      net.bterms.push_back(p);
    }
  }
  for (int g = 0; g < c->n_groups; g++) d.groups.push_back(Group{c->group_name ? c->group_name[g] : sfmt("g%d", g), c->group_visual_debug[g] != 0, c->group_region[g]});
  for (int r = 0; r < c->n_regions; r++) {
    Region reg;
    for (int b = c->region_bound_start[r]; b < c->region_bound_start[r + 1]; b++) reg.boundaries.push_back(rect4(c->region_bounds + 4 * b));
    for (int g = c->region_group_start[r]; g < c->region_group_start[r + 1]; g++) reg.groups.push_back(c->region_groups[g]);
    d.regions.push_back(reg);
  }
  for (int b = 0; b < c->n_blockages; b++) {
    Blockage bl;
    bl.bbox = rect4(c->blockage_box + 4 * b);
    bl.inst = c->blockage_inst[b];
    bl.inst_fixed = c->blockage_inst_fixed[b] != 0;
    if (bl.inst >= 0) bl.inst_name = d.insts[bl.inst].name;
    bl.max_density = c->blockage_max_density[b];
    d.blockages.push_back(bl);
  }
  return d;
}

// ---------------------------------------------------------------- placer_base.rs

// `Instance::extendSizeByScale` (src/placer_base.rs:255-268).
int64_t Instance::extend_size_by_scale(double scale) {
  int64_t old = area();
  if (old == 0) return 0;
  int32_t cxx = cx(), cyy = cy();
  int32_t new_dx = f2i((double)(ux - lx) * scale);
  int32_t new_dy = f2i((double)(uy - ly) * scale);
  lx = cxx - new_dx / 2;
  ux = cxx + new_dx / 2;
  ly = cyy - new_dy / 2;
  uy = cyy + new_dy / 2;
  return area() - old;
}

// `snapOutward` (src/placer_base.rs:271-278).
void Instance::snap_outward(int32_t ox, int32_t oy, int32_t sx, int32_t sy) {
  auto down = [](int32_t v, int32_t o, int32_t s) { return ((v - o) / s) * s + o; };
  auto up = [](int32_t v, int32_t o, int32_t s) { return ((v + s - 1 - o) / s) * s + o; };
  lx = down(lx, ox, sx);
  ly = down(ly, oy, sy);
  ux = up(ux, ox, sx);
  uy = up(uy, oy, sy);
}

static double dbu_to_microns(const Design &d, int32_t v) { return (double)v / (double)d.dbu; }
static double dbu_area_to_microns(const Design &d, int64_t a) { return (double)a / ((double)d.dbu * (double)d.dbu); }

// `PlacerBaseCommon::init` (src/placer_base.rs:301-403).
Common placer_base_common(Log &log, const Design &d, const Vars &v) {
  log.info("GPL", 1, "---- Initialize GPL Main Data Structures");
  log.info("GPL", 2, sfmt("DBU: %d", d.dbu));
  const RowRec *site = nullptr;
  for (auto &r : d.rows)
    if (!r.pad) {
      site = &r;
      break;
    }
  if (!site) log.error("GPL", 305, "Unable to find a site");
  int32_t site_x = site->site_w, site_y = site->site_h;
  if (!d.die.contains(d.core)) log.error("GPL", 118, "core area outside of die.");
  log.info("GPL", 3, sfmt("%-9s ( %6.3f %6.3f ) um", "SiteSize:", dbu_to_microns(d, site_x), dbu_to_microns(d, site_y)));
  log.info("GPL", 4, sfmt("%-9s ( %6.3f %6.3f ) ( %6.3f %6.3f ) um", "CoreBBox:", dbu_to_microns(d, d.core.lx), dbu_to_microns(d, d.core.ly), dbu_to_microns(d, d.core.ux), dbu_to_microns(d, d.core.uy)));
  log.info("GPL", 16, sfmt("Core area:                  %10.3f um^2", dbu_area_to_microns(d, d.core.area())));
  const int32_t ROW_LIMIT = 6;
  Common c;
  c.site_x = site_x;
  c.site_y = site_y;
  for (size_t k = 0; k < d.insts.size(); k++) {
    const DbInst &di = d.insts[k];
    if (!di.core_auto_placeable) continue;
    bool macro_ = di.master_is_block;
    if (!macro_ && di.bbox.dy() > ROW_LIMIT * site_y) {
      macro_ = true;
      log.warn("GPL", 134, sfmt("Master %s is not marked as a BLOCK in LEF but is more than %d rows tall.  It will be treated as a macro.", di.master.c_str(), ROW_LIMIT));
    }
    Instance inst;
    inst.db = (int)k;
    inst.lx = di.bbox.lx;
    inst.ly = di.bbox.ly;
    inst.ux = di.bbox.lx + di.bbox.dx();
    inst.uy = di.bbox.ly + di.bbox.dy();
    inst.fixed = di.fixed;
    inst.macro_ = macro_;
    if (inst.is_place_instance()) {
      inst.lx -= v.pad_left * site_x;
      inst.ux += v.pad_right * site_x;
    }
    if (di.bbox.dy() > d.core.dy()) log.error("GPL", 119, sfmt("instance %s height is larger than core.", di.name.c_str()));
    if (di.bbox.dx() > d.core.dx()) log.error("GPL", 120, sfmt("instance %s width is larger than core.", di.name.c_str()));
    if (inst.fixed) inst.snap_outward(d.core.lx, d.core.ly, site_x, site_y);
    c.insts.push_back(inst);
  }
  auto signal_pins = [&](const Instance &i) -> int64_t { return i.db >= 0 ? d.insts[i.db].signal_pins : 0; };
  int64_t total_signal_pins = 0, movable_area = 0, total_area = 0;
  for (auto &i : c.insts) {
    if (i.db < 0) continue;
    total_area += i.area();
    if (!i.fixed) {
      total_signal_pins += signal_pins(i);
      movable_area += i.area();
    }
  }
  log.info("GPL", 36, sfmt("Movable instances area:     %10.3f um^2", dbu_area_to_microns(d, movable_area)));
  log.info("GPL", 37, sfmt("Total instances area:       %10.3f um^2", dbu_area_to_microns(d, total_area)));
  double avg_density = movable_area > 0 ? (double)total_signal_pins / (double)movable_area : 0.0;
  int64_t total_adjustment_area = 0;
  if (!v.disable_pin_density_adjust) {
    for (auto &i : c.insts) {
      if (!i.fixed && i.db >= 0) {
        int64_t pins = signal_pins(i);
        if (pins > 2 && avg_density > 0.0) {
          double target_area = (double)pins / avg_density;
          double scale = std::sqrt(target_area / (double)i.area());
          scale = std::min(std::max(scale, 0.95), 1.2);  // f64::clamp
          total_adjustment_area += i.extend_size_by_scale(scale);
        }
      }
    }
  }
  log.info("GPL", 35, sfmt("Pin density area adjust:    %10.3f um^2", dbu_area_to_microns(d, total_adjustment_area)));
  int64_t pins = 0;
  for (size_t k = 0; k < d.nets.size(); k++) {
    const DbNet &n = d.nets[k];
    if (!n.signal_or_clock) continue;
    int64_t count = (int64_t)n.iterms.size();
    if (!v.skip_io) {
      for (auto &p : n.bterms)
        if (!p.has_bbox && !v.place_ios) log.error("GPL", 326, sfmt("%s toplevel port is not placed.", p.name.c_str()));
      count += (int64_t)n.bterms.size();
    }
    pins += count;
    c.nets.push_back({(int)k, count});
  }
  c.pins = pins;
  return c;
}

// `getMinMaxIdx` (src/placer_base.rs:406-411).
std::pair<int32_t, int32_t> min_max_idx(int32_t ll, int32_t uu, int32_t core_ll, int32_t site, int32_t mn, int32_t mx) {
  int32_t lower = (ll - core_ll) / site;
  int32_t rem = (uu - core_ll >= site) ? (uu - core_ll) % site : uu - core_ll;
  int32_t upper = rem == 0 ? (uu - core_ll) / site : (uu - core_ll) / site + 1;
  return {std::max(mn, lower), std::min(mx, upper)};
}

enum Site : uint8_t { SITE_BLOCKED, SITE_ROW, SITE_FIXED };

// `initInstsForUnusableSites` (src/placer_base.rs:503-621).
static std::vector<Instance> init_insts_for_unusable_sites(Log &log, const Design &d, const Common &c, const Base &b) {
  Rect rb = b.region_bbox;
  int32_t sx = c.site_x, sy = c.site_y;
  int64_t count_x = rb.dx() / sx, count_y = rb.dy() / sy;
  int32_t cx = (int32_t)count_x, cy = (int32_t)count_y;
  std::vector<uint8_t> grid((size_t)(count_x * count_y), SITE_ROW);
  auto at = [&](int32_t i, int32_t j) { return (size_t)((int64_t)j * count_x + i); };
  auto mark = [&](const Rect &r, uint8_t s) {
    auto [x0, x1] = min_max_idx(r.lx, r.ux, rb.lx, sx, 0, cx);
    auto [y0, y1] = min_max_idx(r.ly, r.uy, rb.ly, sy, 0, cy);
    for (int32_t i = x0; i < x1; i++)
      for (int32_t j = y0; j < y1; j++) grid[at(i, j)] = s;
  };
  if (b.group < 0) {
    std::fill(grid.begin(), grid.end(), SITE_BLOCKED);
    for (auto &r : d.rows) mark(r.box, SITE_ROW);
    for (auto &g : d.groups)
      if (g.region >= 0)
        for (auto &bd : d.regions[g.region].boundaries) mark(bd, SITE_BLOCKED);
  } else {
    const auto &bds = d.regions[d.groups[b.group].region].boundaries;
    if (bds.size() > 1) {
      std::fill(grid.begin(), grid.end(), SITE_BLOCKED);
      for (auto &bd : bds) mark(bd, SITE_ROW);
    }
  }
  for (auto &bl : d.blockages) {
    if (bl.inst >= 0 && !bl.inst_fixed) log.error("GPL", 3, sfmt("Blockages associated with moveable instances  are unsupported and ignored [inst: %s]\n", bl.inst_name.c_str()));
    auto [x0, x1] = min_max_idx(bl.bbox.lx, bl.bbox.ux, rb.lx, sx, 0, cx);
    auto [y0, y1] = min_max_idx(bl.bbox.ly, bl.bbox.uy, rb.ly, sy, 0, cy);
    float filler_density = (100.0f - bl.max_density) / 100.0f;
    int32_t cells = 0, filled = 0;
    for (int32_t j = y0; j < y1; j++)
      for (int32_t i = x0; i < x1; i++) {
        if (cells == 0 || (float)filled / (float)cells <= filler_density) {
          grid[at(i, j)] = SITE_BLOCKED;
          filled++;
        }
        cells++;
      }
  }
  for (auto &inst : c.insts) {
    if (!inst.fixed || inst.db < 0) continue;
    const DbInst &di = d.insts[inst.db];
    bool in_group = b.group < 0 ? (di.group < 0 || d.groups[di.group].visual_debug) : (di.group == b.group && !d.groups[b.group].visual_debug);
    if (!in_group) continue;
    if (inst.macro_ && di.has_halo) {
      Rect h = di.halo;
      Rect r{di.bbox.lx - h.lx, di.bbox.ly - h.ly, di.bbox.ux + h.ux, di.bbox.uy + h.uy};
      auto [x0, x1] = min_max_idx(r.lx, r.ux, rb.lx, sx, 0, cx);
      auto [y0, y1] = min_max_idx(r.ly, r.uy, rb.ly, sy, 0, cy);
      for (int32_t i = x0; i < x1; i++)
        for (int32_t j = y0; j < y1; j++) grid[at(i, j)] = SITE_BLOCKED;
    }
    auto [x0, x1] = min_max_idx(inst.lx, inst.ux, rb.lx, sx, 0, cx);
    auto [y0, y1] = min_max_idx(inst.ly, inst.uy, rb.ly, sy, 0, cy);
    for (int32_t i = x0; i < x1; i++)
      for (int32_t j = y0; j < y1; j++) grid[at(i, j)] = SITE_FIXED;
  }
  std::vector<Instance> dummies;
  for (int32_t j = 0; j < cy; j++) {
    int32_t i = 0;
    while (i < cx) {
      if (grid[at(i, j)] == SITE_BLOCKED) {
        int32_t start = i;
        while (i < cx && grid[at(i, j)] == SITE_BLOCKED) i++;
        int32_t end_x = i;
        int32_t end_y = j + 1;
        while (end_y < cy) {
          bool all = true;
          for (int32_t x = start; x < end_x; x++)
            if (grid[at(x, end_y)] != SITE_BLOCKED) {
              all = false;
              break;
            }
          if (!all) break;
          end_y++;
        }
        for (int32_t y = j; y < end_y; y++)
          for (int32_t x = start; x < end_x; x++) grid[at(x, y)] = SITE_FIXED;
        Instance dm;
        dm.db = -1;
        dm.lx = rb.lx + sx * start;
        dm.ly = rb.ly + sy * j;
        dm.ux = rb.lx + sx * end_x;
        dm.uy = rb.ly + sy * end_y;
        dm.fixed = true;
        dummies.push_back(dm);
      }
      i++;  // the reference's `for` steps past the cell that ended the run
    }
  }
  return dummies;
}

static std::string group_label(const Design &d, int g, const char *top) { return g < 0 ? std::string(top) : d.groups[g].name; }

// `PlacerBase::printInfo` (src/placer_base.rs:624-648).
static void print_info(Log &log, const Design &d, const Common &c, const Base &b, bool check_density) {
  log.info("GPL", 6, sfmt("Number of instances:        %10ld", (long)(b.place_insts.size() + b.fixed_insts.size() + b.dummies.size())));
  log.info("GPL", 7, sfmt("Movable instances:          %10ld", (long)b.place_insts.size()));
  log.info("GPL", 8, sfmt("Fixed instances:            %10ld", (long)b.fixed_insts.size()));
  log.info("GPL", 9, sfmt("Dummy instances:            %10ld", (long)b.dummies.size()));
  log.info("GPL", 10, sfmt("Number of nets:             %10ld", (long)c.nets.size()));
  log.info("GPL", 11, sfmt("Number of pins:             %10ld", (long)c.pins));
  auto m = [&](int32_t v) { return dbu_to_microns(d, v); };
  log.info("GPL", 12, sfmt("%-15s ( %6.3f %6.3f ) ( %6.3f %6.3f ) um", "Die BBox:", m(d.die.lx), m(d.die.ly), m(d.die.ux), m(d.die.uy)));
  Rect r = b.region_bbox;
  log.info("GPL", 13, sfmt("%-15s ( %6.3f %6.3f ) ( %6.3f %6.3f ) um", "Placement BBox:", m(r.lx), m(r.ly), m(r.ux), m(r.uy)));
  float util = (float)b.place_insts_area / (float)(b.region_area - b.non_place_insts_area) * 100.0f;
  log.info("GPL", 14, sfmt("Region name: %s.", group_label(d, b.group, "top-level").c_str()));
  log.info("GPL", 15, sfmt("Region area:                %10.3f um^2", dbu_area_to_microns(d, b.region_area)));
  log.info("GPL", 17, sfmt("Fixed instances area:       %10.3f um^2", dbu_area_to_microns(d, b.non_place_insts_area)));
  log.info("GPL", 18, sfmt("Movable instances area:     %10.3f um^2", dbu_area_to_microns(d, b.place_insts_area)));
  log.info("GPL", 19, sfmt("%-27s %10.3f %%", "Utilization:", (double)util));
  log.info("GPL", 20, sfmt("Standard cells area:        %10.3f um^2", dbu_area_to_microns(d, b.std_insts_area)));
  log.info("GPL", 21, sfmt("Large instances area:       %10.3f um^2", dbu_area_to_microns(d, b.macro_insts_area)));
  if (check_density && (double)util >= 100.1) log.error("GPL", 301, sfmt("Utilization %.3f %% exceeds 100%%.", (double)util));
}

// `PlacerBase::init` (src/placer_base.rs:430-491).
Base placer_base(Log &log, const Design &d, const Common &c, int group, bool check_density) {
  log.info("GPL", 32, sfmt("---- Initialize Region: %s", group_label(d, group, "Top-level").c_str()));
  Rect core = d.core;
  int region = group >= 0 ? d.groups[group].region : -1;
  Base b;
  b.group = group;
  if (region >= 0 && !d.regions[region].boundaries.empty()) {
    const auto &bd = d.regions[region].boundaries;
    Rect bb = bd[0];
    for (size_t i = 1; i < bd.size(); i++) bb = Rect{std::min(bb.lx, bd[i].lx), std::min(bb.ly, bd[i].ly), std::max(bb.ux, bd[i].ux), std::max(bb.uy, bd[i].uy)};
    bb = bb.intersect(core);
    b.region_bbox = bb;
    b.region_area = bb.area();
  } else {
    b.region_bbox = core;
    b.region_area = core.area();
  }
  auto in_this_group = [&](int k) {
    int g = d.insts[k].group;
    if (group < 0) return g < 0 || d.groups[g].visual_debug;
    return g == group && !d.groups[group].visual_debug;
  };
  for (size_t idx = 0; idx < c.insts.size(); idx++) {
    const Instance &inst = c.insts[idx];
    if (inst.db < 0) continue;
    if (inst.fixed) {
      int64_t overlap = 0;
      if (region < 0 || d.regions[region].boundaries.empty()) {
        Rect r{std::max(core.lx, inst.lx), std::max(core.ly, inst.ly), std::min(core.ux, inst.ux), std::min(core.uy, inst.uy)};
        overlap = (r.lx < r.ux && r.ly < r.uy) ? r.area() : 0;
      } else {
        refuse("a fixed instance against a region's boundaries (dbRegion::getOverlapArea) is not modelled");
      }
      if (overlap == 0) continue;
      b.fixed_insts.push_back((int)idx);
      b.non_place_insts_area += overlap;
    } else {
      if (!in_this_group(inst.db)) continue;
      b.place_insts.push_back((int)idx);
      b.place_insts_area += inst.area();
      if (inst.dy() > c.site_y * 6)
        b.macro_insts_area += inst.area();
      else
        b.std_insts_area += inst.area();
    }
  }
  b.dummies = init_insts_for_unusable_sites(log, d, c, b);
  for (auto &dm : b.dummies) b.non_place_insts_area += dm.area();
  print_info(log, d, c, b, check_density);
  return b;
}

// ---------------------------------------------------------------- initial_place.rs

// `dbTransform` (src/initial_place.rs:68-79).
std::pair<int32_t, int32_t> orient_point(int orient, int32_t x, int32_t y) {
  switch (orient) {
    case GPL_R90: return {-y, x};
    case GPL_R180: return {-x, -y};
    case GPL_R270: return {y, -x};
    case GPL_MY: return {-x, y};
    case GPL_MYR90: return {-y, -x};
    case GPL_MX: return {x, -y};
    case GPL_MXR90: return {y, x};
    default: return {x, y};
  }
}

// `Pin::updateCoordi(dbITerm)` (src/initial_place.rs:84-98).
static std::array<int32_t, 4> iterm_pin(const Design &d, int inst, const Term &t) {
  const DbInst &di = d.insts[inst];
  int32_t icx = di.master_w / 2, icy = di.master_h / 2;
  int32_t ox = 0, oy = 0;
  if (t.has_shape) {
    auto [ax, ay] = orient_point(di.orient, t.shape.lx - icx, t.shape.ly - icy);
    auto [bx, by] = orient_point(di.orient, t.shape.ux - icx, t.shape.uy - icy);
    int32_t lx = std::min(ax, bx) + icx, ux = std::max(ax, bx) + icx;
    int32_t ly = std::min(ay, by) + icy, uy = std::max(ay, by) + icy;
    ox = (lx + ux) / 2 - icx;
    oy = (ly + uy) / 2 - icy;
  }
  return {ox, oy, di.bbox.lx + icx + ox, di.bbox.ly + icy + oy};
}

// `pins` (src/initial_place.rs:101-149).
Ip make_pins(const Design &d, const Common &c, const Vars &v) {
  std::vector<int> inst_map(d.insts.size(), -1);
  for (size_t k = 0; k < c.insts.size(); k++)
    if (c.insts[k].db >= 0) inst_map[c.insts[k].db] = (int)k;
  Ip ip;
  for (auto &i : d.insts) ip.db_bbox.push_back(i.bbox);
  ip.inst_pins.resize(c.insts.size());
  for (auto &[net, cnt] : c.nets) {
    const DbNet &n = d.nets[net];
    std::vector<int> list;
    for (auto &t : n.iterms) {
      auto p4 = iterm_pin(d, t.inst, t);
      int pk = (int)ip.pins.size();
      list.push_back(pk);
      if (inst_map[t.inst] >= 0) ip.inst_pins[inst_map[t.inst]].push_back(pk);
      Pin p;
      p.inst = inst_map[t.inst];
      p.off_x = p4[0];
      p.off_y = p4[1];
      p.cx = p4[2];
      p.cy = p4[3];
      ip.pins.push_back(p);
    }
    if (!v.skip_io) {
      for (auto &pt : n.bterms) {
        Rect b = pt.has_bbox ? pt.bbox : Rect{};
        list.push_back((int)ip.pins.size());
        Pin p;
        p.port = true;
        p.movable_io = v.place_ios && !pt.fixed;
        p.cx = (b.lx + b.ux) / 2;
        p.cy = (b.ly + b.uy) / 2;
        ip.pins.push_back(p);
      }
    }
    ip.net_pins.push_back(list);
  }
  std::vector<int> order(ip.pins.size(), 0);
  size_t k = 0;
  for (auto &[net, cnt] : c.nets) {
    const DbNet &n = d.nets[net];
    for (auto &t : n.iterms) order[k++] = t.order;
    if (!v.skip_io) k += n.bterms.size();
  }
  for (auto &pins : ip.inst_pins) std::stable_sort(pins.begin(), pins.end(), [&](int a, int b) { return order[a] < order[b]; });
  for (size_t q = 0; q < c.insts.size(); q++)
    if (!c.insts[q].fixed) ip.place.push_back((int)q);
  return ip;
}

// `Instance::setCenterLocation` with `Pin::updateLocation` (src/initial_place.rs:152-165).
static void set_center_location(Common &c, Ip &ip, int k, int32_t x, int32_t y) {
  Instance &i = c.insts[k];
  int32_t hx = (i.ux - i.lx) / 2, hy = (i.uy - i.ly) / 2;
  i.lx = x - hx;
  i.ly = y - hy;
  i.ux = x + hx;
  i.uy = y + hy;
  int32_t cx = i.cx(), cy = i.cy();
  for (int pk : ip.inst_pins[k]) {
    ip.pins[pk].cx = cx + ip.pins[pk].off_x;
    ip.pins[pk].cy = cy + ip.pins[pk].off_y;
  }
}

static Rect region_box_of(const Design &d, int r) {
  int32_t x0 = INT32_MAX, y0 = INT32_MAX, x1 = INT32_MIN, y1 = INT32_MIN;
  for (auto &b : d.regions[r].boundaries) {
    x0 = std::min(x0, b.lx);
    y0 = std::min(y0, b.ly);
    x1 = std::max(x1, b.ux);
    y1 = std::max(y1, b.uy);
  }
  return Rect{x0, y0, x1, y1};
}

// `placeInstsInitialPositions` (src/initial_place.rs:169-199).
static void place_insts_initial_positions(Log &log, const Design &d, Common &c, Ip &ip, const IpVars &vars) {
  int32_t ccx = (d.core.lx + d.core.ux) / 2, ccy = (d.core.ly + d.core.uy) / 2;
  long region = 0, db = 0, core = 0;
  std::vector<int> place = ip.place;
  for (int k : place) {
    if (c.insts[k].locked) continue;
    const DbInst &di = d.insts[c.insts[k].db];
    int reg = di.group >= 0 ? d.groups[di.group].region : -1;
    if (reg >= 0) {
      Rect b = region_box_of(d, reg);
      set_center_location(c, ip, k, b.ux - (b.ux - b.lx) / 2, b.uy - (b.uy - b.ly) / 2);
      region++;
    } else if (!vars.force_center && di.placed) {
      Rect b = di.bbox;
      set_center_location(c, ip, k, (b.lx + b.ux) / 2, (b.ly + b.uy) / 2);
      db++;
    } else {
      set_center_location(c, ip, k, ccx, ccy);
      core++;
    }
  }
  log.info("GPL", 51, sfmt("Source of initial instance position counters:\n\tOdb location = %ld\tCore center = %ld\tRegion center = %ld", db, core, region));
}

// `updatePinInfo` (src/initial_place.rs:203-252).
static void update_pin_info(Ip &ip) {
  for (auto &p : ip.pins) p.min_x = p.max_x = p.min_y = p.max_y = false;
  for (auto &net : ip.net_pins) {
    int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
    int pminx = -1, pminy = -1, pmaxx = -1, pmaxy = -1;
    for (int k : net) {
      if (ip.pins[k].movable_io) continue;
      int32_t cx = ip.pins[k].cx, cy = ip.pins[k].cy;
      if (lx > cx) {
        if (pminx >= 0) ip.pins[pminx].min_x = false;
        lx = cx;
        pminx = k;
        ip.pins[k].min_x = true;
      }
      if (ux < cx) {
        if (pmaxx >= 0) ip.pins[pmaxx].max_x = false;
        ux = cx;
        pmaxx = k;
        ip.pins[k].max_x = true;
      }
      if (ly > cy) {
        if (pminy >= 0) ip.pins[pminy].min_y = false;
        ly = cy;
        pminy = k;
        ip.pins[k].min_y = true;
      }
      if (uy < cy) {
        if (pmaxy >= 0) ip.pins[pmaxy].max_y = false;
        uy = cy;
        pmaxy = k;
        ip.pins[k].max_y = true;
      }
    }
  }
}

struct System {
  std::vector<std::tuple<int64_t, int64_t, float>> triplets;
  std::vector<float> rhs, x;
};

// `createSparseMatrix` (src/initial_place.rs:264-355).
static void create_sparse_matrix(const Common &c, const Ip &ip, const IpVars &vars, System &sx, System &sy) {
  size_t n = ip.place.size();
  std::vector<int64_t> ext(c.insts.size(), -1);
  for (size_t e = 0; e < n; e++) ext[ip.place[e]] = (int64_t)e;
  sx.triplets.clear();
  sy.triplets.clear();
  sx.rhs.assign(n, 0.0f);
  sy.rhs.assign(n, 0.0f);
  sx.x.assign(n, 0.0f);
  sy.x.assign(n, 0.0f);
  for (size_t e = 0; e < n; e++) {
    int k = ip.place[e];
    sx.x[e] = (float)c.insts[k].cx();
    sy.x[e] = (float)c.insts[k].cy();
    if (c.insts[k].locked) {
      sx.triplets.emplace_back(e, e, 1.0f);
      sy.triplets.emplace_back(e, e, 1.0f);
      sx.rhs[e] = (float)c.insts[k].cx();
      sy.rhs[e] = (float)c.insts[k].cy();
    }
  }
  auto placed = [&](const Pin &p) -> int { return (p.inst >= 0 && !c.insts[p.inst].fixed) ? p.inst : -1; };
  std::vector<int> solve;
  for (auto &net : ip.net_pins) {
    if (net.size() <= 1 || (int)net.size() >= vars.max_fanout) continue;
    float net_weight = vars.net_weight_scale / (float)(net.size() - 1);
    solve.clear();
    for (int k : net)
      if (!ip.pins[k].movable_io) solve.push_back(k);
    for (size_t i1 = 1; i1 < solve.size(); i1++) {
      const Pin &p1 = ip.pins[solve[i1]];
      for (size_t i2 = 0; i2 < i1; i2++) {
        const Pin &p2 = ip.pins[solve[i2]];
        if (p1.inst == p2.inst) continue;
        for (int axis = 0; axis < 2; axis++) {
          bool marked;
          int32_t c1, c2;
          System *sys;
          if (axis == 0) {
            marked = p1.min_x || p1.max_x || p2.min_x || p2.max_x;
            c1 = p1.cx;
            c2 = p2.cx;
            sys = &sx;
          } else {
            marked = p1.min_y || p1.max_y || p2.min_y || p2.max_y;
            c1 = p1.cy;
            c2 = p2.cy;
            sys = &sy;
          }
          if (!marked) continue;
          auto center = [&](int k) { return axis == 0 ? c.insts[k].cx() : c.insts[k].cy(); };
          int32_t diff = std::abs(c1 - c2);
          float weight = diff > vars.min_diff_length ? net_weight / (float)diff : net_weight / (float)vars.min_diff_length;
          int a = placed(p1), bb = placed(p2);
          if (a >= 0 && bb >= 0) {
            bool la = c.insts[a].locked, lb = c.insts[bb].locked;
            if (!la && !lb) {
              int64_t e1 = ext[a], e2 = ext[bb];
              sys->triplets.emplace_back(e1, e1, weight);
              sys->triplets.emplace_back(e2, e2, weight);
              sys->triplets.emplace_back(e1, e2, -weight);
              sys->triplets.emplace_back(e2, e1, -weight);
              sys->rhs[e1] += -weight * (float)((c1 - center(a)) - (c2 - center(bb)));
              sys->rhs[e2] += -weight * (float)((c2 - center(bb)) - (c1 - center(a)));
            } else if (la && !lb) {
              int64_t e2 = ext[bb];
              sys->triplets.emplace_back(e2, e2, weight);
              sys->rhs[e2] += weight * (float)(c1 - (c2 - center(bb)));
            } else if (!la && lb) {
              int64_t e1 = ext[a];
              sys->triplets.emplace_back(e1, e1, weight);
              sys->rhs[e1] += weight * (float)(c2 - (c1 - center(a)));
            }
          } else if (a < 0 && bb >= 0) {
            int64_t e2 = ext[bb];
            sys->triplets.emplace_back(e2, e2, weight);
            sys->rhs[e2] += weight * (float)(c1 - (c2 - center(bb)));
          } else if (a >= 0 && bb < 0) {
            int64_t e1 = ext[a];
            sys->triplets.emplace_back(e1, e1, weight);
            sys->rhs[e1] += weight * (float)(c2 - (c1 - center(a)));
          }
        }
      }
    }
  }
}

// `hpwl` over the database boxes (src/initial_place.rs:359-386).
static int64_t ip_hpwl(const Design &d, const Common &c, const Ip &ip, const Vars &v) {
  int64_t total = 0;
  for (auto &[net, cnt] : c.nets) {
    const DbNet &n = d.nets[net];
    int32_t lx = INT32_MAX, ly = INT32_MAX, ux = INT32_MIN, uy = INT32_MIN;
    for (auto &t : n.iterms) {
      Rect b = ip.db_bbox[t.inst];
      lx = std::min(lx, b.lx);
      ly = std::min(ly, b.ly);
      ux = std::max(ux, b.ux);
      uy = std::max(uy, b.uy);
    }
    if (!v.skip_io)
      for (auto &p : n.bterms)
        if (p.has_bbox) {
          lx = std::min(lx, p.bbox.lx);
          ly = std::min(ly, p.bbox.ly);
          ux = std::max(ux, p.bbox.ux);
          uy = std::max(uy, p.bbox.uy);
        }
    if (ux >= lx) total += (int64_t)(ux - lx) + (int64_t)(uy - ly);
  }
  return total;
}

// `updateCoordi` (src/initial_place.rs:391-417).
static void update_coordi(const Design &d, Common &c, Ip &ip, const std::vector<float> &sx, const std::vector<float> &sy) {
  std::vector<int> place = ip.place;
  for (size_t e = 0; e < place.size(); e++) {
    int k = place[e];
    if (c.insts[k].locked) continue;
    int32_t nx = f2i(sx[e]), ny = f2i(sy[e]);
    nx = std::min(std::max(nx, d.core.lx), d.core.ux);
    ny = std::min(std::max(ny, d.core.ly), d.core.uy);
    int di = c.insts[k].db;
    int g = d.insts[di].group;
    if (g >= 0 && d.groups[g].region >= 0) {
      Rect b = region_box_of(d, d.groups[g].region);
      nx = std::min(std::max(nx, b.lx), b.ux);
      ny = std::min(std::max(ny, b.ly), b.uy);
    }
    set_center_location(c, ip, k, nx, ny);
    int32_t lx = c.insts[k].lx, ly = c.insts[k].ly;
    Rect b = ip.db_bbox[di];
    ip.db_bbox[di] = Rect{lx, ly, lx + b.dx(), ly + b.dy()};
  }
}

static uint64_t fnv_f32(const std::vector<float> &v) {
  uint64_t h = 1469598103934665603ull;
  for (float f : v) {
    uint32_t b;
    std::memcpy(&b, &f, 4);
    for (int i = 0; i < 4; i++) {
      h ^= (b >> (8 * i)) & 0xff;
      h *= 1099511628211ull;
    }
  }
  return h;
}

// `doBicgstabPlace` (src/initial_place.rs:420-446).
Ip do_bicgstab_place(Log &log, const Design &d, Common &c, const Vars &v, const IpVars &vars) {
  log.info("GPL", 5, "---- Execute Conjugate Gradient Initial Placement.");
  Ip ip = make_pins(d, c, v);
  place_insts_initial_positions(log, d, c, ip, vars);
  System sx, sy;
  for (int iter = 1; iter <= vars.max_iter; iter++) {
    update_pin_info(ip);
    create_sparse_matrix(c, ip, vars, sx, sy);
    int64_t n = (int64_t)ip.place.size();
    Csr mx = Csr::from_triplets(n, sx.triplets);
    Solve ex = bicgstab(mx, sx.rhs, sx.x, vars.max_solver_iter);
    Csr my = Csr::from_triplets(n, sy.triplets);
    Solve ey = bicgstab(my, sy.rhs, sy.x, vars.max_solver_iter);
    uint32_t exb, eyb;
    std::memcpy(&exb, &ex.error, 4);
    std::memcpy(&eyb, &ey.error, 4);
    log.probe(sfmt("VYGIPS|%d|x|%d|%08x|%d|%016llx", iter, ex.iterations, exb, ex.converged ? 0 : 2, (unsigned long long)fnv_f32(sx.x)));
    log.probe(sfmt("VYGIPS|%d|y|%d|%08x|%d|%016llx", iter, ey.iterations, eyb, ey.converged ? 0 : 2, (unsigned long long)fnv_f32(sy.x)));
    if (std::isnan(ex.error) || std::isnan(ey.error)) {
      log.warn("GPL", 325, sfmt("Conjugate gradient initial placement solver failed at iteration %d. ", iter));
      break;
    }
    float error_max = fmaxr(ex.error, ey.error);
    log.report(sfmt("[InitialPlace]  Iter: %d conjugate gradient residual: %.8f HPWL: %ld", iter, (double)error_max, (long)ip_hpwl(d, c, ip, v)));
    update_coordi(d, c, ip, sx.x, sy.x);
    if ((double)error_max <= 1e-5 && iter >= 5) break;
  }
  return ip;
}

// ---------------------------------------------------------------- bicgstab.rs

// `Csr::from_triplets` (src/bicgstab.rs:501-541): duplicates summed per column in triplet
// order into the first occurrence, then rows in column order.
Csr Csr::from_triplets(int64_t n, const std::vector<std::tuple<int64_t, int64_t, float>> &t) {
  // bucket the triplets by column, keeping their order
  std::vector<int64_t> cstart(n + 1, 0);
  for (auto &[r, cc, v] : t) cstart[cc + 1]++;
  for (int64_t i = 0; i < n; i++) cstart[i + 1] += cstart[i];
  std::vector<int64_t> fill(cstart.begin(), cstart.end() - 1);
  std::vector<std::pair<int64_t, float>> bycol(t.size());
  for (auto &[r, cc, v] : t) bycol[fill[cc]++] = {r, v};
  // collapse duplicates per column
  std::vector<int64_t> slot(n, -1);
  std::vector<std::vector<std::pair<int64_t, float>>> collapsed(n);
  for (int64_t cc = 0; cc < n; cc++) {
    auto &out = collapsed[cc];
    for (int64_t q = cstart[cc]; q < cstart[cc + 1]; q++) {
      auto [r, v] = bycol[q];
      if (slot[r] >= 0)
        out[slot[r]].second += v;
      else {
        slot[r] = (int64_t)out.size();
        out.push_back({r, v});
      }
    }
    for (auto &e : out) slot[e.first] = -1;
  }
  // transposed copy: rows in column order
  Csr m;
  m.n = n;
  std::vector<int64_t> rcount(n + 1, 0);
  for (int64_t cc = 0; cc < n; cc++)
    for (auto &e : collapsed[cc]) rcount[e.first + 1]++;
  for (int64_t i = 0; i < n; i++) rcount[i + 1] += rcount[i];
  m.starts = rcount;
  m.cols.resize(rcount[n]);
  m.vals.resize(rcount[n]);
  std::vector<int64_t> rf(rcount.begin(), rcount.end() - 1);
  for (int64_t cc = 0; cc < n; cc++)
    for (auto &e : collapsed[cc]) {
      m.cols[rf[e.first]] = (int32_t)cc;
      m.vals[rf[e.first]++] = e.second;
    }
  return m;
}

// `Csr::mul` (src/bicgstab.rs:544-554).
void Csr::mul(const float *x, float *y) const {
  for (int64_t i = 0; i < n; i++) {
    float tmp = 0.0f;
    for (int64_t k = starts[i]; k < starts[i + 1]; k++) tmp += vals[k] * x[cols[k]];
    y[i] = 0.0f + 1.0f * tmp;
  }
}

// `sum` (src/bicgstab.rs:559-595): Eigen's SSE2 packet order. With ORACLE_SUM_DOUBLE=1 in the
// environment the terms are instead summed in double, in index order, and the total rounded to
// float once: a measurement of how far the rounding of the inner products alone moves a run (the
// device forms them in double), never a parity reference.
static bool sum_in_double() {
  static const bool on = [] {
    const char *e = std::getenv("ORACLE_SUM_DOUBLE");
    return e && e[0] == '1';
  }();
  return on;
}
float eigen_sum(int64_t n, const float *a, const float *b) {
  auto f = [&](int64_t i) -> float { return b ? a[i] * b[i] : a[i]; };
  if (sum_in_double()) {
    double acc = 0.0;
    for (int64_t i = 0; i < n; i++) acc += b ? (double)a[i] * (double)b[i] : (double)a[i];
    return (float)acc;
  }
  const int64_t P = 4;
  int64_t aligned_size2 = (n / (2 * P)) * (2 * P);
  int64_t aligned_size = (n / P) * P;
  if (aligned_size == 0) {
    if (n == 0) return 0.0f;
    float res = f(0);
    for (int64_t i = 1; i < n; i++) res += f(i);
    return res;
  }
  float p0[4] = {f(0), f(1), f(2), f(3)};
  if (aligned_size > P) {
    float p1[4] = {f(4), f(5), f(6), f(7)};
    for (int64_t i = 2 * P; i < aligned_size2; i += 2 * P) {
      for (int q = 0; q < 4; q++) p0[q] = p0[q] + f(i + q);
      for (int q = 0; q < 4; q++) p1[q] = p1[q] + f(i + P + q);
    }
    for (int q = 0; q < 4; q++) p0[q] = p0[q] + p1[q];
    if (aligned_size > aligned_size2)
      for (int q = 0; q < 4; q++) p0[q] = p0[q] + f(aligned_size2 + q);
  }
  float res = (p0[0] + p0[2]) + (p0[1] + p0[3]);
  for (int64_t i = aligned_size; i < n; i++) res += f(i);
  return res;
}

// `bicgstab` (src/bicgstab.rs:615-669), float throughout, the library's order.
Solve bicgstab(const Csr &mat, const std::vector<float> &rhs, std::vector<float> &x, int max_iters) {
  const float tol = 1.1920929e-07f;  // f32::EPSILON
  int64_t n = mat.n;
  std::vector<float> mx(n), r(n), r0, v(n, 0.0f), p(n, 0.0f), y, s(n), z, t(n);
  mat.mul(x.data(), mx.data());
  for (int64_t i = 0; i < n; i++) r[i] = rhs[i] - mx[i];
  r0 = r;
  float r0_sqnorm = eigen_sum(n, r0.data(), r0.data());
  float rhs_sqnorm = eigen_sum(n, rhs.data(), rhs.data());
  if (rhs_sqnorm == 0.0f) {
    std::fill(x.begin(), x.end(), 0.0f);
    return Solve{max_iters, tol, true};
  }
  float rho = 1.0f, alpha = 1.0f, w = 1.0f;
  float tol2 = tol * tol * rhs_sqnorm;
  float eps2 = tol * tol;
  int i = 0, restarts = 0;
  while (eigen_sum(n, r.data(), r.data()) > tol2 && i < max_iters) {
    float rho_old = rho;
    rho = eigen_sum(n, r0.data(), r.data());
    if (std::fabs(rho) < eps2 * r0_sqnorm) {
      mat.mul(x.data(), mx.data());
      for (int64_t k = 0; k < n; k++) r[k] = rhs[k] - mx[k];
      r0 = r;
      r0_sqnorm = eigen_sum(n, r.data(), r.data());
      rho = r0_sqnorm;
      if (restarts == 0) i = 0;
      restarts++;
    }
    float beta = (rho / rho_old) * (alpha / w);
    for (int64_t k = 0; k < n; k++) p[k] = r[k] + beta * (p[k] - w * v[k]);
    y = p;
    mat.mul(y.data(), v.data());
    alpha = rho / eigen_sum(n, r0.data(), v.data());
    for (int64_t k = 0; k < n; k++) s[k] = r[k] - alpha * v[k];
    z = s;
    mat.mul(z.data(), t.data());
    float tmp = eigen_sum(n, t.data(), t.data());
    w = tmp > 0.0f ? eigen_sum(n, t.data(), s.data()) / tmp : 0.0f;
    for (int64_t k = 0; k < n; k++) x[k] += alpha * y[k] + w * z[k];
    for (int64_t k = 0; k < n; k++) r[k] = s[k] - w * t[k];
    i++;
  }
  float error = std::sqrt(eigen_sum(n, r.data(), r.data()) / rhs_sqnorm);
  return Solve{i, error, error <= tol};
}

// ---------------------------------------------------------------- normal.rs

// `Mt19937::new` (src/normal.rs:50-77): init_genrand, then the library's word-0 fix-up.
Mt19937::Mt19937(uint32_t seed) {
  x[0] = seed;
  for (int k = 1; k < 624; k++) x[k] = 1812433253u * (x[k - 1] ^ (x[k - 1] >> 30)) + (uint32_t)k;
  i = 624;
  uint32_t y0 = x[396] ^ x[623];
  if (y0 & 0x80000000u)
    y0 = ((y0 ^ 0x9908b0dfu) << 1) | 1;
  else
    y0 <<= 1;
  x[0] = (x[0] & 0x80000000u) | (y0 & 0x7fffffffu);
  bool all0 = true;
  for (int k = 0; k < 624; k++)
    if (x[k]) {
      all0 = false;
      break;
    }
  if (all0) x[0] = 0x80000000u;
}

void Mt19937::twist() {
  const uint32_t A = 0x9908b0dfu, U = 0x80000000u, L = 0x7fffffffu;
  for (int j = 0; j < 624 - 397; j++) {
    uint32_t y = (x[j] & U) | (x[j + 1] & L);
    x[j] = x[j + 397] ^ (y >> 1) ^ ((x[j + 1] & 1u) * A);
  }
  for (int j = 624 - 397; j < 623; j++) {
    uint32_t y = (x[j] & U) | (x[j + 1] & L);
    x[j] = x[j - (624 - 397)] ^ (y >> 1) ^ ((x[j + 1] & 1u) * A);
  }
  uint32_t y = (x[623] & U) | (x[0] & L);
  x[623] = x[396] ^ (y >> 1) ^ ((x[0] & 1u) * A);
  i = 0;
}

uint32_t Mt19937::next_u32() {
  if (i == 624) twist();
  uint32_t z = x[i++];
  z ^= z >> 11;
  z ^= (z << 7) & 0x9d2c5680u;
  z ^= (z << 15) & 0xefc60000u;
  z ^= z >> 18;
  return z;
}

// `uniform_int` (src/normal.rs:108-127).
int32_t uniform_int(Mt19937 &eng, int32_t mn, int32_t mx) {
  uint32_t range = (uint32_t)((int64_t)mx - (int64_t)mn);
  if (range == 0) return mn;
  const uint32_t brange = UINT32_MAX;
  if (range == brange) return (int32_t)((int64_t)mn + (int64_t)eng.next_u32());
  uint32_t bucket = brange / (range + 1);
  if (brange % (range + 1) == range) bucket++;
  while (true) {
    uint32_t r = eng.next_u32() / bucket;
    if (r <= range) return (int32_t)((int64_t)mn + (int64_t)r);
  }
}

static double tbl(const uint64_t *t, int i) {
  double v;
  std::memcpy(&v, &t[i], 8);
  return v;
}
#define NX(i) tbl(kNORMALX_BITS, (i))
#define NY(i) tbl(kNORMALY_BITS, (i))
#define EX(i) tbl(kEXPX_BITS, (i))
#define EY(i) tbl(kEXPY_BITS, (i))

// `int_float_pair` (src/normal.rs:137-145).
static double int_float_pair(Mt19937 &eng, int &bucket) {
  uint32_t u = eng.next_u32();
  bucket = (int)(u & 0xff);
  double r = (double)(u >> 8) * (1.0 / (double)(1u << 24));
  u = eng.next_u32();
  r += (double)(u & 0x1fffffffu);
  r *= 0.5 / (double)(1u << 28);
  return r;
}
static double uniform_01(Mt19937 &eng) {
  double factor = 1.0 / ((double)UINT32_MAX + 1.0);
  return (double)eng.next_u32() * factor;
}
// `unit_exponential` (src/normal.rs:197-214).
static double unit_exponential(Mt19937 &eng) {
  double shift = 0.0;
  while (true) {
    int i;
    double r = int_float_pair(eng, i);
    double x = r * EX(i);
    if (x < EX(i + 1)) return shift + x;
    if (i == 0) {
      shift += EX(1);
    } else {
      double y01 = uniform_01(eng);
      double y = EY(i) + y01 * (EY(i + 1) - EY(i));
      double above_ubound = (EX(i) - EX(i + 1)) * y01 - (EX(i) - x);
      double above_lbound = y - (EY(i + 1) + (EX(i + 1) - x) * EY(i + 1));
      if (above_ubound < 0.0 && (above_lbound < 0.0 || y < std::exp(-x))) return x + shift;
    }
  }
}
// `normal_tail` (src/normal.rs:184-193).
static double normal_tail(Mt19937 &eng) {
  double tail_start = NX(1);
  while (true) {
    double x = unit_exponential(eng) / tail_start;
    double y = unit_exponential(eng) / 1.0;
    if (2.0 * y > x * x) return x + tail_start;
  }
}
// `unit_normal` (src/normal.rs:154-179).
static double unit_normal(Mt19937 &eng) {
  while (true) {
    int bucket;
    double r = int_float_pair(eng, bucket);
    double sign = (double)((bucket & 1) * 2 - 1);
    int i = bucket >> 1;
    double x = r * NX(i);
    if (x < NX(i + 1)) return x * sign;
    if (i == 0) return normal_tail(eng) * sign;
    double y01 = uniform_01(eng);
    double y = NY(i) + y01 * (NY(i + 1) - NY(i));
    double chord = (NX(i) - NX(i + 1)) * y01 - (NX(i) - x);
    double tangent = y - (NY(i) + (NX(i) - x) * NY(i) * NX(i));
    double above_ubound, above_lbound;
    if (NX(i) >= 1.0) {
      above_ubound = chord;
      above_lbound = tangent;
    } else {
      above_ubound = tangent;
      above_lbound = chord;
    }
    if (above_ubound < 0.0 && (above_lbound < 0.0 || y < std::exp(-(x * x / 2.0)))) return x * sign;
  }
}
// `normal` (src/normal.rs:131-133).
double normal(Mt19937 &eng, double mean, double sigma) { return unit_normal(eng) * sigma + mean; }

}  // namespace orc
