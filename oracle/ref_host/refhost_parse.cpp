/*
 * Oracle A, project-input side: the reference's own parser
 * (V_02_2015/src/Input/KSimulationData.cpp, compiled unmodified beside this
 * file) wrapped in one C entry point, so tests can compare the product's
 * project-input mirror against it and the golden-fixture generator can read
 * the reference's fixtures exactly as the reference does.  TEST
 * INFRASTRUCTURE ONLY.
 *
 * KSimulationData opens "../Projects/<project>/World/<world>.World" relative
 * to the working directory (KSimulationData.cpp:33-56), so the caller passes
 * a run directory whose parent holds a Projects/ tree (a scratch copy: the
 * parser also writes a log file into the project folder).
 */
#include <cstring>
#include <string>
#include <unistd.h>

#include "Input/KSimulationData.h"

extern "C" {

/* Plain-old-data image of everything the parser's getters return
 * (KSimulationData.h:32-75) that the simulation-step setup uses. */
struct RefProject {
  int particle_type, sim_type, read_file, num_particles;
  int n_w, n_p, n_d, num_lifters, is_debug, is_rotation;
  int per_object[16];
  float delta_t, roll_res, global_damp, vel_limit;
  float3 gravity, grid_origin, grid_size, world_size;
  char filename[256];
  Mill_Data mill;
  Silo_Data silo;
  InitConfig init;
};

int refh_project_sizeof(void) { return (int)sizeof(RefProject); }

int refh_parse(const char* run_dir, const char* project, const char* world, RefProject* out,
               WOBJ* w_out, int w_cap, POBJ* p_out, int p_cap, DOBJ* d_out, int d_cap) {
  char old[4096];
  if (!getcwd(old, sizeof(old))) return 10;
  if (chdir(run_dir) != 0) return 11;
  KSimulationData* k = new KSimulationData(project, world);
  int rc = chdir(old) != 0 ? 12 : 0;
  std::memset(out, 0, sizeof(RefProject));
  out->particle_type = k->get_particleType();
  out->sim_type = k->get_simType();
  out->read_file = k->get_readFile();
  out->num_particles = k->get_num_Particles();
  out->n_w = k->get_num_WorldObjects();
  out->n_p = k->get_num_ParticleObjects();
  out->n_d = k->get_num_DYParticleObjects();
  out->num_lifters = k->get_num_Lifters();
  out->is_debug = k->get_isDebug();
  out->is_rotation = k->get_isRotation();
  for (int i = 0; i < 16 && i < out->n_p; ++i) out->per_object[i] = k->get_num_ParticlesPerObject()[i];
  out->delta_t = k->get_delta_t();
  out->roll_res = k->get_RollRes();
  out->global_damp = k->get_GlobalDamp();
  out->vel_limit = k->get_velLimit();
  out->gravity = k->get_gravity();
  out->grid_origin = k->get_NNGrid().origin;
  out->grid_size = k->get_NNGrid().size;
  out->world_size = k->get_worldSize();
  std::string fn = k->get_filename();
  std::strncpy(out->filename, fn.c_str(), sizeof(out->filename) - 1);
  out->mill = k->get_millObject();
  out->silo = k->get_siloObject();
  out->init = k->get_InitPosGrid();
  if (out->n_w > w_cap || out->n_p > p_cap || out->n_d > d_cap) return 13;
  std::memcpy(w_out, k->get_worldObject(), sizeof(WOBJ) * out->n_w);
  std::memcpy(p_out, k->get_particleObject(), sizeof(POBJ) * out->n_p);
  if (out->n_d > 0) std::memcpy(d_out, k->get_dynamicObject(), sizeof(DOBJ) * out->n_d);
  return rc;
}

}  // extern "C"
