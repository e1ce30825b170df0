"""ctypes images of the POD types that cross the simulation-step boundary.

Field order and types follow include/blaze_types.h, which in turn follows the
reference's V_02_2015/src/DataStructures/KSimulationObjects.h:104-381 and
V_02_2015/src/Utilities/Common/Types.h:15-21.  ctypes applies the same
natural-alignment rules as the C compiler, so sizes and offsets match; the
CPU test-suite checks them against the reference's headers.
"""
import ctypes as C

c_bool = C.c_bool


class float3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]

    def __iter__(self):
        return iter((self.x, self.y, self.z))

    def set(self, v):
        self.x, self.y, self.z = (float(v[0]), float(v[1]), float(v[2]))
        return self


class int3(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("z", C.c_int)]


class Quaterion(C.Structure):
    _fields_ = [("w", C.c_float), ("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class SimulationInfo(C.Structure):
    _fields_ = [
        ("particle_type", C.c_int),
        ("Num_Particles", C.c_int),
        ("Num_ParticleObjects", C.c_int),
        ("Num_ParticlesPerObject", C.POINTER(C.c_int)),
        ("Num_WorldObjects", C.c_int),
        ("TotnumCells", C.c_int),
        ("Rotation", c_bool),
        ("Mode2D", c_bool),
        ("EnergyCalc", c_bool),
        ("isMillSim", c_bool),
        ("Kill_Particles", c_bool),
        ("InitalDelta_t", C.c_float),
        ("MillRotVel", C.c_float),
        ("Global_VisDamp", C.c_float),
        ("Roll_Res", C.c_float),
        ("Silo_Kill_Height", C.c_float),
        ("Vel_Limit", C.c_float),
        ("DObject_CylinderBoundR", C.c_float),
        ("num_NNCells", int3),
        ("Force_Field", float3),
        ("worldOrigin", float3),
        ("cellSize", float3),
        ("cent", float3),
        ("Vel_Limit_Bounds", float3),
        ("max_size", float3),
        ("Simulation_Type", C.c_int),
        ("Integration_Type", C.c_int),
        ("use_symmetry", c_bool),
        ("sphere_orient", c_bool),
        ("dobject_hasVertex", c_bool),
        ("Rotating_WObject", c_bool),
        ("use_hist", c_bool),
        ("unit_test", C.c_int),
    ]


class InitConfig(C.Structure):
    _fields_ = [
        ("num", int3),
        ("space", float3),
        ("start", float3),
        ("p_size", float3 * 16),
        ("is_spheres", c_bool),
        ("use_file", c_bool),
        ("grid_type", C.c_int),
        ("launch_Vel", float3),
        ("fill_plane_start", float3),
        ("fill_plane_end", float3),
        ("velocity", float3 * 12),
        ("position", float3 * 12),
        ("ang_vel", float3 * 12),
        ("DebugFlag", c_bool),
        ("use_device", C.c_int),
        ("multi_gpu", c_bool),
        ("threads_perBlock", C.c_int),
    ]


class Edge_Def(C.Structure):
    _fields_ = [("point_vindex", C.c_uint * 2)]


class Surface(C.Structure):
    _fields_ = [
        ("num_vertex", C.c_int),
        ("vertex_Order", C.c_int * 8),
        ("area", C.c_float),
        ("normal", float3),
        ("centroid", float3),
        ("Tol", C.c_float),
    ]


class PP_Parms(C.Structure):
    _fields_ = [("Kn", C.c_float), ("Cn", C.c_float),
                ("Fric_static", C.c_float), ("Fric_kinetic", C.c_float)]


class POBJ(C.Structure):
    _fields_ = [
        ("radius", C.c_float),
        ("mass", C.c_float),
        ("COM", float3),
        ("num_vertex", C.c_int),
        ("Local_Vertex", float3 * 32),
        ("num_edges", C.c_int),
        ("edge", Edge_Def * 32),
        ("num_faces", C.c_int),
        ("face", Surface * 32),
        ("InertiaT", C.c_float * 9),
        ("vertex", float3 * 32),
        ("PP", PP_Parms * 6),
        ("surface_Kn", C.c_float),
        ("surface_Cn", C.c_float),
        ("surface_Fric_static", C.c_float),
        ("surface_Fric_kinetic", C.c_float),
        ("Dsurface_Kn", C.c_float),
        ("Dsurface_Cn", C.c_float),
        ("Dsurface_Fric_static", C.c_float),
        ("Dsurface_Fric_kinetic", C.c_float),
    ]


class DOBJ(C.Structure):
    _fields_ = [
        ("btype", C.c_uint),
        ("Axis", float3),
        ("boundR", C.c_float),
        ("COM", float3),
        ("num_vertex", C.c_int),
        ("vertex", float3 * 8),
        ("num_faces", C.c_int),
        ("faces", Surface * 3),
        ("num_edges", C.c_int),
        ("edge", Edge_Def * 4),
        ("velocity", float3),
        ("is_attached_DWorld", c_bool),
        ("is_translating", c_bool),
    ]


class Macro_Cylinder(C.Structure):
    _fields_ = [
        ("height", C.c_float),
        ("radius", C.c_float),
        ("has_top_cap", c_bool),
        ("has_bot_cap", c_bool),
        ("normal_cyl", float3),
        ("normal_top_cap", float3),
        ("normal_bot_cap", float3),
        ("center_top_cap", float3),
        ("center_bot_cap", float3),
        ("AXIS", float3),
    ]


class WOBJ(C.Structure):
    _fields_ = [
        ("surface_type", C.c_int),
        ("num_surfaces", C.c_int),
        ("surfaces", Surface * 16),
        ("num_vertex", C.c_int),
        ("vertex", float3 * 16),
        ("is_rotating", c_bool),
        ("cyl_geo", Macro_Cylinder),
    ]


class Mill_Data(C.Structure):
    """KSimulationObjects.h:60-69 (host-side project data, not sent to the device)."""
    _fields_ = [
        ("power_output_revs", C.c_int),
        ("total_revs", C.c_int),
        ("mill_RPM", C.c_float),
        ("RadPerStep", C.c_double),
        ("Num_Steps_PerRev", C.c_int),
        ("Rot_PerStep", C.c_int),
        ("Current_StepNumber", C.c_int),
    ]


class Silo_Data(C.Structure):
    """KSimulationObjects.h:71-83."""
    _fields_ = [
        ("measure_flow", c_bool),
        ("flow_steps", C.c_int),
        ("kill_particle", c_bool),
        ("is_hatch_open", c_bool),
        ("manual_hatch", c_bool),
        ("flow_count", C.c_int),
        ("num_particles_rem", C.c_int),
        ("hatch_height", C.c_float),
        ("flow_rate", C.c_int),
    ]


BOUNDARY_TYPES = {
    "SimulationInfo": SimulationInfo,
    "POBJ": POBJ,
    "WOBJ": WOBJ,
    "DOBJ": DOBJ,
    "InitConfig": InitConfig,
    "Surface": Surface,
    "Macro_Cylinder": Macro_Cylinder,
    "PP_Parms": PP_Parms,
    "Quaterion": Quaterion,
}
