// state_writer.cu -- the reference's state-file format on the host
// (Output_SystemState, FileIO.h:12-315): a header line by detail level and
// particle kind, "Specfication_Detail: d", a simulation line (mill:
// revolution, time, angle, tallies; silo: time, particles left; rotating
// world object: time, steps, angle; otherwise time), one row per particle
// still in the run (P_ID != -1) in memory order, then the mean and largest
// speed (m/s; a silo counts the particles above the hatch) and, for a mill,
// the power line.  Numbers go through std::ostream with its default
// formatting and the same insertions, so the files read back the same way
// the reference's do (Read_FromFile, FileIO.h:327-652).
#include <cmath>
#include <fstream>
#include <vector>

#include "blaze_dem.h"

namespace {

struct V3 { float x, y, z; };

inline V3 at3(const float* a, int i) { return V3{a[3 * i], a[3 * i + 1], a[3 * i + 2]}; }
// length(v * 0.010) of the host operators: each component times 0.01f, sqrtf
// of the dot product in x, y, z order
inline float speed_ms(V3 v) {
  const float s = 0.010f;
  const float x = v.x * s, y = v.y * s, z = v.z * s;
  return sqrtf(x * x + y * y + z * z);
}

const char* header_line(int detail, bool poly) {
  switch (detail) {
    case 1:
      return poly ? "#  P_ID    PType_ID   Pos(x,y,z)cm  Orient(w,x,y,z)"
                  : "#  P_ID    PType_ID   Pos(x,y,z)cm  ";
    case 2:
      return poly ? "#  P_ID   PType_ID   Pos(x,y,z)cm    Vel(x,y,z)cm/s  Orient(w,x,y,z) AngVel(x,y,z)cm/s"
                  : "#  P_ID   PType_ID   Pos(x,y,z)cm    Vel(x,y,z)cm/s    AngVel(x,y,z)cm/s";
    case 3:
      return poly ? "#  P_ID   PType_ID   Pos(x,y,z)cm  Vel(x,y,z)cm/s    Orient(w,x,y,z)  AngVel(x,y,z)cm/s"
                  : "#  P_ID   PType_ID   Pos(x,y,z)cm  Vel(x,y,z)cm/s     AngVel(x,y,z)cm/s";
    case 4:
      return poly ? "#  P_ID   PType_ID   Pos(x,y,z)cm  Vel(x,y,z)cm/s    Orient(w,x,y,z)  AngVel(x,y,z)cm/s  | MagVel(m/s)  MagAVel(m/s)"
                  : "#  P_ID   PType_ID   Pos(x,y,z)cm  Vel(x,y,z)cm/s    AngVel(x,y,z)cm/s   | MagVel(m/s)  MagAVel(m/s) ";
    case 5:
      return "# COM   Vertex";
    default:
      return nullptr;
  }
}

}  // namespace

extern "C" int blaze_write_state_arrays(const char* path, const blaze_state_header* h, int n,
                                        const float* pos3, const float* quat4, const float* vel3,
                                        const float* avel3, const float* acc3, const uint* type,
                                        const int* pid, const POBJ* pobj, int n_p) {
  if (!path || !h || n < 0 || !pos3 || !type || !pid) return -1;
  const int d = h->detail;
  const bool poly = h->particle_type == 1;
  if (d < 1 || d > 5) return -1;
  if (d >= 2 && (!vel3 || !avel3)) return -1;
  if (d == 4 && !acc3) return -1;
  if (poly && d <= 4 && !quat4) return -1;
  if (d == 5 && !pobj) return -1;
  std::ofstream out(path);
  if (!out) return -3;
  out << header_line(d, poly) << std::endl;
  out << "Specfication_Detail: " << d << std::endl;
  if (h->sim_type == 1) {
    int rev = h->rev_number;
    if (h->revflag == 0) rev--;
    else rev++;
    if (h->fill_start) {
      out << " RevNum: " << 0 << "  Time: " << 0.0 << " RevComplete: " << 0 << "  RotAngle: "
          << h->rot_angle << "  EParticle: " << 0.0 << " ELift " << 0.0 << " EDrum: " << 0.0
          << " ENorm: " << 0.0 << " EShear: " << 0.0 << std::endl;
    } else {
      out << " RevNum: " << rev << "  Time: " << h->time << " RevComplete: " << h->revflag
          << "  RotAngle: " << h->rot_angle << "  EParticle: " << h->energy[0] << " ELift "
          << h->energy[1] << " EDrum: " << h->energy[2] << " ENorm: " << h->energy[3]
          << " EShear: " << h->energy[4] << std::endl;
    }
  } else if (h->sim_type == 2) {
    out << "  Time: " << h->time << " NumRem: " << h->num_rem << std::endl;
  } else if (h->rotating_wobj) {
    out << "  Time: " << h->time << "  RotSteps: " << h->rot_steps << "  RotAngle: "
        << h->rot_angle << std::endl;
  } else {
    out << "  Time: " << h->time << std::endl;
  }
  int silo_count = 0;
  float sumV = 0.0f, maxVel = 0.0f;
  int maxID = -1;
  for (int i = 0; i < n; ++i) {
    if (pid[i] == -1) continue;
    const V3 p = at3(pos3, i);
    if (d == 1) {
      out << pid[i] << "  " << type[i] << "    " << p.x << "  " << p.y << "  " << p.z << "    ";
      if (!poly) out << std::endl;
      else
        out << quat4[4 * i] << "  " << quat4[4 * i + 1] << "  " << quat4[4 * i + 2] << "  "
            << quat4[4 * i + 3] << std::endl;
    } else if (d == 2 || d == 3 || d == 4) {
      const V3 v = at3(vel3, i), w = at3(avel3, i);
      if (d == 2)
        out << pid[i] << "  " << type[i] << "    " << p.x << "  " << p.y << "  " << p.z << "    "
            << v.x << "  " << v.y << "  " << v.z;
      else if (d == 3)
        out << pid[i] << "  " << type[i] << "    " << p.x << " " << p.y << " " << p.z
            << "       " << v.x << "   " << v.y << "   " << v.z;
      else
        out << pid[i] << "  " << type[i] << "    " << p.x << " " << p.y << " " << p.z
            << "      " << "       " << v.x << "   " << v.y << "   " << v.z;
      if (poly) {
        out << (d == 2 ? "    " : "       ") << quat4[4 * i] << (d == 2 ? "   " : "   ")
            << quat4[4 * i + 1] << "   " << quat4[4 * i + 2] << " " << quat4[4 * i + 3];
      }
      out << "       " << w.x << "   " << w.y << "   " << w.z;
      if (d == 4) {
        out << "       " << speed_ms(v) << "   " << speed_ms(w) << "   "
            << speed_ms(at3(acc3, i));
      }
      out << std::endl;
    } else {  // d == 5: the object's vertices about the particle
      out << pid[i] << "  " << type[i] << "    " << p.x << " " << p.y << " " << p.z << "      ";
      const int t = (int)type[i];
      if (t >= 0 && t < n_p) {
        const POBJ& o = pobj[t];
        for (int k = 0; k < o.num_vertex && k < 32; ++k) {
          const float3 q = o.vertex[k];
          out << (q.x + p.x) << "  " << (q.y + p.y) << "  " << (q.z + p.z) << "    ";
        }
      }
      out << std::endl;
    }
    const float sp = vel3 ? speed_ms(at3(vel3, i)) : 0.0f;
    if (h->sim_type == 2) {
      if (p.y > h->hatch_height) {
        silo_count++;
        sumV += sp;
        if (sp > maxVel) { maxVel = sp; maxID = pid[i]; }
      }
    } else {
      sumV += sp;
      if (sp > maxVel) { maxVel = sp; maxID = pid[i]; }
    }
  }
  if (h->sim_type == 2) out << "# Average Vel(m/s) " << sumV / silo_count << std::endl;
  else out << "# Average Vel(m/s) " << sumV / n << std::endl;
  out << "# MAXVEL (m/s) " << maxVel << " Particle " << maxID << std::endl;
  if (h->sim_type == 1) {
    const float per = (float)h->steps_per_rev * h->dt;
    out << "# RevNum: " << h->rev_number << "  Time(s): " << h->time << " Power(W): "
        << ((h->energy[0] + h->energy[2]) / per) << std::endl;
  }
  return out.good() ? 0 : -3;
}

// The driver's result files, one line per call, appended, with the
// reference's expressions and ostream's default formatting.
//
// FlowRate.dat of a silo run (main.cpp:133-147): every flow_steps steps
// after the hatch opens, the time and the percentage discharged,
// (n0 - remaining) / (float) n0 * 100, remaining counted as Silo_Stats
// counts it (blaze_count_above).
extern "C" int blaze_write_flow_line(const char* path, double time, int n0, int remaining) {
  if (!path || n0 <= 0) return -1;
  std::ofstream out(path, std::ios::app);
  if (!out) return -3;
  out << time << " " << ((n0 - remaining) / (float)n0) * 100.0 << std::endl;
  return out.good() ? 0 : -3;
}

// Results.dat of a ball-mill run (main.cpp:53-82): at the end of every
// revolution the power from the energy tallies of that revolution
// (Device_Get_Energy's three values: particle, lifter, drum).
extern "C" int blaze_write_power_line(const char* path, double time, const float* energy3,
                                      int steps_per_rev, float dt) {
  if (!path || !energy3) return -1;
  std::ofstream out(path, std::ios::app);
  if (!out) return -3;
  const float* e = energy3;
  out << "time: " << time << " Power:   Total = " << ((e[0] + e[1] + e[2]) / (steps_per_rev * dt))
      << "  Particle: " << (e[0]) / (steps_per_rev * dt)
      << "  Lifter: " << e[1] / (steps_per_rev * dt) << " Drum " << e[2] / (steps_per_rev * dt)
      << std::endl;
  return out.good() ? 0 : -3;
}
