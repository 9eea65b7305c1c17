// C entry points of the scene builder and the error channel shared by every entry point of the library.
#include <algorithm>
#include <cstring>
#include <exception>
#include <string>

#include "errors.hpp"
#include "host_goals.hpp"
#include "scene.hpp"

namespace wsb {
static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }
const std::string &last_error() { return g_last_error; }
}  // namespace wsb

extern "C" {

int ws_last_error(char *buf, size_t n) {
  const std::string &e = wsb::last_error();
  if (buf && n) {
    size_t k = std::min(n - 1, e.size());
    std::memcpy(buf, e.data(), k);
    buf[k] = 0;
  }
  return int(e.size());
}

// params.js:8-23 in SI: strength 1e4 N/mm -> 1e7 N/m, epsilon 15 mm -> 0.015 m
void ws_params_default(ws_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->mass_scale = 1.5; p->damping = 1.0; p->tol = 1e-4; p->kinetic_damping = 1; p->warmup_iter = 300; p->max_iter = 5000;
  p->contacts = 1; p->strength = 1e7; p->stick_strength = 1e7; p->torsion_factor = 1.0; p->epsilon = 0.015;
  p->ramp_iter = 1500; p->slip_rate = 1.0; p->edge_threshold = 0.5;
  p->augmented = 0; p->al_every = 600; p->rot_friction = 0; p->seat_law = 0; p->seat_gap = 1; p->dent_after_iter = -1;
  p->rot_factor = 1.0; p->dent_rate = 0.01;
  p->floor = 0; p->floor_z = 0.0; p->floor_mu = 0.5;
}

int ws_scene_kagome(const ws_kagome_cfg *cfg, ws_scene **out) {
  if (!cfg || !out) return wsb::fail(WS_ERR_ARG, "ws_scene_kagome: null argument");
  try {
    wsb::Scene *sc = wsb::buildKagome(*cfg);
    *out = new ws_scene{sc};
    return WS_OK;
  } catch (const std::exception &e) { return wsb::fail(WS_ERR_ARG, std::string("ws_scene_kagome: ") + e.what()); }
}

int ws_scene_mesh(const ws_mesh_cfg *cfg, ws_scene **out) {
  if (!cfg || !out) return wsb::fail(WS_ERR_ARG, "ws_scene_mesh: null argument");
  try {
    wsb::Scene *sc = wsb::buildMeshScene(*cfg);
    *out = new ws_scene{sc};
    return WS_OK;
  } catch (const std::exception &e) { return wsb::fail(WS_ERR_ARG, std::string("ws_scene_mesh: ") + e.what()); }
}

int ws_scene_polylines(const ws_polyline_cfg *cfg, ws_scene **out) {
  if (!cfg || !out) return wsb::fail(WS_ERR_ARG, "ws_scene_polylines: null argument");
  try {
    wsb::Scene *sc = wsb::buildPolylineScene(*cfg);
    *out = new ws_scene{sc};
    return WS_OK;
  } catch (const std::exception &e) { return wsb::fail(WS_ERR_ARG, std::string("ws_scene_polylines: ") + e.what()); }
}

const ws_model *ws_scene_model(const ws_scene *s) { return s ? &s->sc->model : nullptr; }
const int32_t *ws_scene_node_offset(const ws_scene *s) { return s ? s->sc->st.nodeOffset.data() : nullptr; }
double ws_scene_span(const ws_scene *s) { return s ? s->sc->span() : 0.0; }
int ws_model_goals(const ws_model *md, double *mass, double *krs, double *u, double *nprev, double *l_ref) {
  if (!md) return wsb::fail(WS_ERR_ARG, "ws_model_goals: null model");
  try {
    wsb::HostGoals g;
    g.build(*md);
    if (mass) std::copy(g.mass.begin(), g.mass.end(), mass);
    if (krs) std::copy(g.kRotStatic.begin(), g.kRotStatic.end(), krs);
    if (u) std::copy(g.u.begin(), g.u.end(), u);
    if (nprev) std::copy(g.nPrev.begin(), g.nPrev.end(), nprev);
    if (l_ref) *l_ref = g.lRef;
    return WS_OK;
  } catch (const std::exception &e) { return wsb::fail(WS_ERR_ARG, std::string("ws_model_goals: ") + e.what()); }
}

void ws_scene_free(ws_scene *s) {
  if (!s) return;
  delete s->sc;
  delete s;
}

}  // extern "C"
