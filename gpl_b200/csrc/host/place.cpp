// Host side, part 1: the logger and its formats, the design records, the placer's
// construction (src/placer_base.rs), the initial placement's host half (src/initial_place.rs:
// pins, start points, the B2B matrix assembly, the CSR build of src/bicgstab.rs:501-541) with
// the solve itself on the device, and the random numbers (src/normal.rs) the Nesterov setup
// draws.
#include <algorithm>
#include <atomic>
#include <charconv>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <tuple>

#include "host.h"
#include "parallel.h"
#include "../kernels/b2b.h"

namespace gpl {

#include "ziggurat_tables.inc"

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

// An instance's (or its master's) name, generated as "i<k>" ("m<k>") when the caller gave none.
std::string inst_label(const Design &d, size_t k) { return d.insts[k].name.empty() ? sfmt("i%zu", k) : d.insts[k].name; }
std::string master_label(const Design &d, size_t k) { return d.insts[k].master.empty() ? sfmt("m%zu", k) : d.insts[k].master; }

Design design_from_c(const gpl_design_t *c) {
  Design d;
  d.dbu = c->dbu;
  d.die = rect4(c->die);
  d.core = rect4(c->core);
  for (int r = 0; r < c->n_rows; r++) d.rows.push_back(RowRec{rect4(c->row_box + 4 * r), c->row_pad[r] != 0, c->row_site[2 * r], c->row_site[2 * r + 1]});
  big_resize(d.insts, (size_t)std::max(c->n_insts, 0));
  parallel_for((size_t)std::max(c->n_insts, 0), [&](size_t k0, size_t k1) {
    for (int k = (int)k0; k < (int)k1; k++) {
      DbInst &i = d.insts[k];
      // names the caller did not give are generated when a message needs them (inst_label)
      if (c->inst_name) i.name = c->inst_name[k];
      if (c->inst_master_name) i.master = c->inst_master_name[k];
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
  });
  big_resize(d.nets, (size_t)std::max(c->n_nets, 0));
  parallel_for((size_t)std::max(c->n_nets, 0), [&](size_t n0, size_t n1) {
    for (int n = (int)n0; n < (int)n1; n++) {
      DbNet &net = d.nets[n];
      if (c->net_name) net.name = c->net_name[n];
      net.signal_or_clock = c->net_signal[n] != 0;
      net.iterms.reserve((size_t)(c->net_iterm_start[n + 1] - c->net_iterm_start[n]));
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
  });
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
    if (bl.inst >= 0) bl.inst_name = inst_label(d, bl.inst);
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
  c.insts.reserve(d.insts.size());
  c.nets.reserve(d.nets.size());
  for (size_t k = 0; k < d.insts.size(); k++) {
    const DbInst &di = d.insts[k];
    if (!di.core_auto_placeable) continue;
    bool macro_ = di.master_is_block;
    if (!macro_ && di.bbox.dy() > ROW_LIMIT * site_y) {
      macro_ = true;
      log.warn("GPL", 134, sfmt("Master %s is not marked as a BLOCK in LEF but is more than %d rows tall.  It will be treated as a macro.", master_label(d, k).c_str(), ROW_LIMIT));
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
    if (di.bbox.dy() > d.core.dy()) log.error("GPL", 119, sfmt("instance %s height is larger than core.", inst_label(d, k).c_str()));
    if (di.bbox.dx() > d.core.dx()) log.error("GPL", 120, sfmt("instance %s width is larger than core.", inst_label(d, k).c_str()));
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
  // each instance grows by its own pin count alone: the instances go in parallel, and the
  // total is an integer sum
  std::atomic<int64_t> total_adjustment_area{0};
  if (!v.disable_pin_density_adjust) {
    parallel_for(c.insts.size(), [&](size_t a, size_t b) {
      int64_t part = 0;
      for (size_t k = a; k < b; k++) {
        Instance &i = c.insts[k];
        if (!i.fixed && i.db >= 0) {
          int64_t pins = signal_pins(i);
          if (pins > 2 && avg_density > 0.0) {
            double target_area = (double)pins / avg_density;
            double scale = std::sqrt(target_area / (double)i.area());
            scale = std::min(std::max(scale, 0.95), 1.2);  // f64::clamp
            part += i.extend_size_by_scale(scale);
          }
        }
      }
      total_adjustment_area += part;
    });
  }
  log.info("GPL", 35, sfmt("Pin density area adjust:    %10.3f um^2", dbu_area_to_microns(d, total_adjustment_area.load())));
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
  big_resize(ip.db_bbox, d.insts.size());
  parallel_for(d.insts.size(), [&](size_t a, size_t b) {
    for (size_t i = a; i < b; i++) ip.db_bbox[i] = d.insts[i].bbox;
  });
  // sized up front: pins are made net by net, so net n's pins are the run of pin numbers
  // from its start; each instance's list is counted first
  const size_t nn = c.nets.size();
  ip.net_pins.start.assign(nn + 1, 0);
  ip.inst_pins.start.assign(c.insts.size() + 1, 0);
  // the counts in parallel (an instance's count by atomic adds: a sum, whatever their order),
  // then the two scans
  int64_t *inst_count = ip.inst_pins.start.data();
  parallel_for(nn, [&](size_t a, size_t b) {
    for (size_t n = a; n < b; n++) {
      const DbNet &dn = d.nets[c.nets[n].first];
      ip.net_pins.start[n + 1] = (int64_t)(dn.iterms.size() + (v.skip_io ? 0 : dn.bterms.size()));
      for (auto &t : dn.iterms)
        if (inst_map[t.inst] >= 0) __atomic_fetch_add(&inst_count[inst_map[t.inst] + 1], (int64_t)1, __ATOMIC_RELAXED);
    }
  });
  for (size_t n = 0; n < nn; n++) ip.net_pins.start[n + 1] += ip.net_pins.start[n];
  const size_t total = (size_t)ip.net_pins.start[nn];
  for (size_t k = 0; k < c.insts.size(); k++) ip.inst_pins.start[k + 1] += ip.inst_pins.start[k];
  progress("    pins: counted");
  big_resize(ip.net_pins.items, total);
  big_resize(ip.pins, total);
  std::vector<int> order;
  big_assign(order, total, 0);
  progress("    pins: arrays sized");
  parallel_for(nn, [&](size_t a, size_t b) {
    for (size_t n = a; n < b; n++) {
      const DbNet &dn = d.nets[c.nets[n].first];
      int64_t pk = ip.net_pins.start[n];
      for (auto &t : dn.iterms) {
        auto p4 = iterm_pin(d, t.inst, t);
        Pin &p = ip.pins[pk];
        p.inst = inst_map[t.inst];
        p.off_x = p4[0];
        p.off_y = p4[1];
        p.cx = p4[2];
        p.cy = p4[3];
        order[pk] = t.order;
        ip.net_pins.items[pk] = (int)pk;
        pk++;
      }
      if (!v.skip_io) {
        for (auto &pt : dn.bterms) {
          Rect r = pt.has_bbox ? pt.bbox : Rect{};
          Pin &p = ip.pins[pk];
          p.port = true;
          p.movable_io = v.place_ios && !pt.fixed;
          p.cx = (r.lx + r.ux) / 2;
          p.cy = (r.ly + r.uy) / 2;
          ip.net_pins.items[pk] = (int)pk;
          pk++;
        }
      }
    }
  });
  progress("    pins: made");
  // each instance's pins in its iterms' order (the reference walks an instance's iterms),
  // ties in pin (net) order: the lists are filled in parallel in any order, then each sorted
  // by (iterm order, pin), which is the net-order fill's stable sort by iterm order
  big_resize(ip.inst_pins.items, (size_t)ip.inst_pins.start.back());
  std::vector<int64_t> fill(ip.inst_pins.start.begin(), ip.inst_pins.start.end() - 1);
  parallel_for(total, [&](size_t a, size_t b) {
    for (size_t q = a; q < b; q++) {
      int k = ip.pins[q].inst;
      if (k >= 0 && !ip.pins[q].port) ip.inst_pins.items[__atomic_fetch_add(&fill[k], (int64_t)1, __ATOMIC_RELAXED)] = (int)q;
    }
  });
  progress("    pins: instance lists filled");
  auto by_order = [&](int x, int y) { return order[x] < order[y] || (order[x] == order[y] && x < y); };
  parallel_for(c.insts.size(), [&](size_t a, size_t b) {
    for (size_t q = a; q < b; q++) {
      int *lo = ip.inst_pins.begin_of(q), *hi = ip.inst_pins.end_of(q);
      if (!std::is_sorted(lo, hi, by_order)) std::sort(lo, hi, by_order);
    }
  });
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
  // each instance moves with its own pins only, so the instances go in parallel; the
  // counters are summed over the chunks
  std::atomic<long> region{0}, db{0}, core{0};
  const std::vector<int> &place = ip.place;
  parallel_for(place.size(), [&](size_t a, size_t b) {
    long n_region = 0, n_db = 0, n_core = 0;
    for (size_t e = a; e < b; e++) {
      const int k = place[e];
      if (c.insts[k].locked) continue;
      const DbInst &di = d.insts[c.insts[k].db];
      int reg = di.group >= 0 ? d.groups[di.group].region : -1;
      if (reg >= 0) {
        Rect r = region_box_of(d, reg);
        set_center_location(c, ip, k, r.ux - (r.ux - r.lx) / 2, r.uy - (r.uy - r.ly) / 2);
        n_region++;
      } else if (!vars.force_center && di.placed) {
        Rect r = di.bbox;
        set_center_location(c, ip, k, (r.lx + r.ux) / 2, (r.ly + r.uy) / 2);
        n_db++;
      } else {
        set_center_location(c, ip, k, ccx, ccy);
        n_core++;
      }
    }
    region += n_region;
    db += n_db;
    core += n_core;
  });
  log.info("GPL", 51, sfmt("Source of initial instance position counters:\n\tOdb location = %ld\tCore center = %ld\tRegion center = %ld", db.load(), core.load(), region.load()));
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

// `doBicgstabPlace` (src/initial_place.rs:420-446) with its matrices assembled, collapsed and
// solved on the device (kernels/b2b.cu): the reference's rounds, report lines, probes and stop
// rules; the host reads back the two solves' scalars and the report's HPWL per round.
Ip do_bicgstab_place_device(Log &log, const Design &d, Common &c, const Vars &v, const IpVars &vars, IpDevice &dev) {
  log.info("GPL", 5, "---- Execute Conjugate Gradient Initial Placement.");
  Ip ip = make_pins(d, c, v);
  progress("pins made");
  place_insts_initial_positions(log, d, c, ip, vars);
  if (vars.max_iter < 1) return ip;
  auto device = [](cudaError_t e, const char *where) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("device: ") + cudaGetErrorString(e) + " in " + where);
  };
  // the device's view: placed instances in `ip.place` order, pins net by net
  IpSetup s;
  const size_t n = ip.place.size();
  std::vector<int32_t> ext(c.insts.size(), -1);
  for (size_t e = 0; e < n; e++) ext[ip.place[e]] = (int32_t)e;
  s.core = make_int4(d.core.lx, d.core.ly, d.core.ux, d.core.uy);
  big_resize(s.box, n);
  big_resize(s.locked, n);
  big_resize(s.grouped, n);
  big_resize(s.clamp, n);
  big_resize(s.db_box, n);
  big_resize(s.db_size, n);
  parallel_for(n, [&](size_t a, size_t b) {
    for (size_t e = a; e < b; e++) {
      const Instance &i = c.insts[ip.place[e]];
      s.box[e] = make_int4(i.lx, i.ly, i.ux, i.uy);
      s.locked[e] = i.locked ? 1 : 0;
      int g = d.insts[i.db].group;
      bool grouped = g >= 0 && d.groups[g].region >= 0;
      Rect r = grouped ? region_box_of(d, d.groups[g].region) : Rect{};
      s.grouped[e] = grouped ? 1 : 0;
      s.clamp[e] = make_int4(r.lx, r.ly, r.ux, r.uy);
      Rect bb = ip.db_bbox[i.db];
      s.db_box[e] = make_int4(bb.lx, bb.ly, bb.ux, bb.uy);
      s.db_size[e] = make_int2(bb.dx(), bb.dy());
    }
  });
  std::vector<int> inst_map(d.insts.size(), -1);
  for (size_t k = 0; k < c.insts.size(); k++)
    if (c.insts[k].db >= 0) inst_map[c.insts[k].db] = (int)k;
  progress("    set-up: instances");
  // pins net by net, as make_pins numbered them (net n's run starts at net_pins.start[n])
  const size_t np = ip.pins.size(), nn = c.nets.size();
  if (ip.net_pins.size() != nn || (size_t)ip.net_pins.start[nn] != np) throw std::runtime_error("initial placement: pin order mismatch");
  big_resize(s.pin_e, np);
  big_resize(s.pin_inst, np);
  big_resize(s.pin_mio, np);
  big_resize(s.pin_off, np);
  big_resize(s.pin_xy, np);
  big_resize(s.pin_hp, np);
  big_resize(s.pin_static, np);
  s.net_start.assign(ip.net_pins.start.begin(), ip.net_pins.start.end());
  progress("    set-up: pin arrays sized");
  parallel_for(nn, [&](size_t a, size_t b) {
    for (size_t ni = a; ni < b; ni++) {
      const DbNet &dn = d.nets[c.nets[ni].first];
      size_t pk = (size_t)ip.net_pins.start[ni];
      for (auto &t : dn.iterms) {
        const Pin &p = ip.pins[pk];
        int k = inst_map[t.inst];
        bool placed = p.inst >= 0 && !c.insts[p.inst].fixed;
        s.pin_e[pk] = placed ? ext[p.inst] : -1;
        s.pin_inst[pk] = p.inst;
        s.pin_mio[pk] = p.movable_io ? 1 : 0;
        s.pin_off[pk] = make_int2(p.off_x, p.off_y);
        s.pin_xy[pk] = make_int2(p.cx, p.cy);
        bool dynamic = k >= 0 && !c.insts[k].fixed;
        Rect bb = ip.db_bbox[t.inst];
        s.pin_hp[pk] = dynamic ? 0 : 1;
        s.pin_static[pk] = make_int4(bb.lx, bb.ly, bb.ux, bb.uy);
        pk++;
      }
      if (!v.skip_io)
        for (auto &pt : dn.bterms) {
          const Pin &p = ip.pins[pk];
          s.pin_e[pk] = -1;
          s.pin_inst[pk] = p.inst;
          s.pin_mio[pk] = p.movable_io ? 1 : 0;
          s.pin_off[pk] = make_int2(p.off_x, p.off_y);
          s.pin_xy[pk] = make_int2(p.cx, p.cy);
          s.pin_hp[pk] = pt.has_bbox ? 1 : 2;
          s.pin_static[pk] = make_int4(pt.bbox.lx, pt.bbox.ly, pt.bbox.ux, pt.bbox.uy);
          pk++;
        }
    }
  });

  progress("initial placement set up on the host");
  s.max_fanout = vars.max_fanout;
  s.min_diff = vars.min_diff_length;
  s.weight_scale = vars.net_weight_scale;
  device(dev.upload(s), "initial placement upload");
  progress("initial placement (device): %zu pins, %zu nets", ip.pins.size(), ip.net_pins.size());
  std::vector<float> xs, ys;
  for (int iter = 1; iter <= vars.max_iter; iter++) {
    IpAxisResult r[2];
    device(dev.assemble(r), "initial placement assembly");
    progress("  round %d: B2B assembled and collapsed (%lld + %lld triplets)", iter, (long long)r[0].triplets, (long long)r[1].triplets);
    device(dev.solve(vars.max_solver_iter, r), "initial placement solves");
    const BicgResult &ex = r[0].solve, &ey = r[1].solve;
    progress("  round %d: solved (%d + %d iterations)", iter, ex.iterations, ey.iterations);
    if (log.trace_on) {
      device(dev.solution(0, xs), "initial placement solution");
      device(dev.solution(1, ys), "initial placement solution");
    }
    uint32_t exb, eyb;
    std::memcpy(&exb, &ex.error, 4);
    std::memcpy(&eyb, &ey.error, 4);
    log.probe(sfmt("VYGIPS|%d|x|%d|%08x|%d|%016llx", iter, ex.iterations, exb, ex.converged ? 0 : 2, (unsigned long long)fnv_f32(xs)));
    log.probe(sfmt("VYGIPS|%d|y|%d|%08x|%d|%016llx", iter, ey.iterations, eyb, ey.converged ? 0 : 2, (unsigned long long)fnv_f32(ys)));
    if (std::isnan(ex.error) || std::isnan(ey.error)) {
      log.warn("GPL", 325, sfmt("Conjugate gradient initial placement solver failed at iteration %d. ", iter));
      break;
    }
    float error_max = fmaxr(ex.error, ey.error);
    int64_t hp = 0;
    device(dev.hpwl(&hp), "initial placement hpwl");
    log.report(sfmt("[InitialPlace]  Iter: %d conjugate gradient residual: %.8f HPWL: %ld", iter, (double)error_max, (long)hp));
    device(dev.update(), "initial placement update");
    if ((double)error_max <= 1e-5 && iter >= 5) break;
  }
  progress("initial placement rounds done (%s)", dev.tuning().c_str());
  // the placed instances, their database boxes and their pins back on the host
  std::vector<int4> box, db_box;
  device(dev.download(box, db_box), "initial placement download");
  progress("initial placement downloaded");
  // each placed instance writes only itself, its database box and its own pins
  parallel_for(n, [&](size_t a, size_t b) {
    for (size_t e = a; e < b; e++) {
      int k = ip.place[e];
      Instance &i = c.insts[k];
      if (i.locked) continue;
      i.lx = box[e].x;
      i.ly = box[e].y;
      i.ux = box[e].z;
      i.uy = box[e].w;
      ip.db_bbox[i.db] = Rect{db_box[e].x, db_box[e].y, db_box[e].z, db_box[e].w};
      int32_t cx = i.cx(), cy = i.cy();
      for (int q : ip.inst_pins[k]) {
        ip.pins[q].cx = cx + ip.pins[q].off_x;
        ip.pins[q].cy = cy + ip.pins[q].off_y;
      }
    }
  });
  return ip;
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

}  // namespace gpl

#include <chrono>
#include <cstdlib>
namespace gpl {
void progress(const char *fmt, ...) {
  static const bool on = std::getenv("GPL_LOG") != nullptr;
  static const auto t0 = std::chrono::steady_clock::now();
  if (!on) return;
  double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  std::fprintf(stderr, "[gpl %9.3f] %s\n", s, buf);
  std::fflush(stderr);
}
}  // namespace gpl
