/*
 * fdtd_c.h — C-ABI of the B200 FDTD time-stepping library (libfdtd_b200.so).
 *
 * The reference exposes this path as the C++ class interface of PML_WaveSolver
 * (src/wavesolver/PML_WaveSolver.h:122-255) driven by FDTD_AcousticSimulator
 * (src/wavesolver/FDTD_AcousticSimulator.cpp:419-621) and SimWorld::StepWorld
 * (src/wavesolver/SimWorld.cpp:507-592).  Each entry point below names the
 * reference member it replaces.  Signatures use plain pointers and sizes only;
 * no exception crosses this boundary: every call returns an fdtd_status and the
 * message of the last failure is kept per handle (fdtd_solver_last_error) and
 * per thread (fdtd_last_error).
 *
 * Units are SI (m, s, kg/m^3).  Flat cell index is i*Ny*Nz + j*Nz + k with z
 * contiguous (src/field/ScalarField.cpp:86-97).
 */
#ifndef FDTD_C_H
#define FDTD_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FDTD_ABI_VERSION 5

typedef int32_t fdtd_status;
enum {
    FDTD_OK = 0,
    FDTD_END_OF_TIME = 1,          /* stepSystem() returning false at endTime (PML_WaveSolver.cpp:605-606) */
    FDTD_ERR_INVALID_ARG = -1,     /* std::runtime_error on bad input */
    FDTD_ERR_OOM = -2,
    FDTD_ERR_CUDA = -3,
    FDTD_ERR_NUMERIC = -4,         /* NaN/Inf seen in a listener series */
    FDTD_ERR_TIMEOUT = -5,         /* a bounded device wait ran out */
    FDTD_ERR_GEOMETRY = -6,        /* fresh cell inside an object (MAC_Grid.cpp:2050-2053) */
    FDTD_ERR_UNSUPPORTED = -7,     /* a reference feature outside this library's scope */
    FDTD_ERR_IO = -8,
    FDTD_ERR_BUSY = -9,            /* server queue full / slot table full */
    FDTD_ERR_CANCELLED = -10       /* the request was cancelled (fdtd_server_cancel) */
};

/* ---------------------------------------------------------------------------
 * Scene description (plain data, copied at create time)
 * ------------------------------------------------------------------------- */
enum { FDTD_SHAPE_SPHERE = 0, FDTD_SHAPE_BOX = 1, FDTD_SHAPE_ELLIPSOID = 2,
       FDTD_SHAPE_MESH = 3 /* closed triangle mesh (FDTD_RigidObject over a surface .obj) */ };

/* A closed, consistently oriented triangle mesh in its object frame (the
 * reference's FDTD_RigidObject::_mesh after MeshObjReader's scaling,
 * FDTD_RigidObject.cpp:84-93): world = rotation * v + center.  Triangles are
 * counter-clockwise seen from outside; every edge must be shared by exactly two
 * triangles (the signed distance field of FDTD_RigidObject.cpp:59-76 rejects
 * meshes with a boundary). */
typedef struct {
    int32_t n_vertices;
    int32_t n_triangles;
    const double* vertices;    /* 3 * n_vertices                                        */
    const int32_t* triangles;  /* 3 * n_triangles vertex indices                        */
} fdtd_mesh_desc;

/* Boundary normal-acceleration model of an object (replaces the vibrational
 * sources summed by FDTD_RigidObject::EvaluateBoundaryAcceleration,
 * src/wavesolver/FDTD_RigidObject.cpp:330-368).  g(t) = A*exp(-((t-t0)/tau)^2/2). */
enum {
    FDTD_ACCEL_NONE = 0,
    FDTD_ACCEL_GAUSSIAN_TRANSLATION = 1, /* a(x,t) = g(t) * dir (rigid translation)       */
    FDTD_ACCEL_GAUSSIAN_PULSATION = 2    /* a(x,t) = g(t) * n(x) (sphere only, monopole) */
};

enum {
    FDTD_MOTION_STATIC = 0,
    FDTD_MOTION_BALLISTIC = 1,
    /* keyframes (fdtd_keyframe_track): centre of mass lerped and rotation slerped
     * between frames, FDTD_RigidObject_Blender_Animator::GetRigidObjectTransform
     * (FDTD_RigidObject_Animator.cpp:128-155) and FDTD_RigidObject::
     * SetRigidBodyTransform (FDTD_RigidObject.cpp:549-566): the body's local origin
     * goes to the frame's centre and its rest rotation is turned by the frame's */
    FDTD_MOTION_KEYFRAMED = 2
};

/* Keyframes of one FDTD_MOTION_KEYFRAMED object: frame i at time i * step, with
 * frames[7 i .. 7 i + 6] = centre x, y, z and rotation quaternion w, x, y, z
 * (a kinematics file of FDTD_RigidObject_Animator.cpp:79-122 after its y-up
 * correction; fdtd_read_kinematics reads one).  Before the first frame the first
 * holds, after the last the last. */
typedef struct {
    int32_t object;          /* index into fdtd_scene_desc.objects */
    int32_t n_frames;
    double step;             /* seconds between frames (1 / kinematics_frame_rate) */
    const double* frames;    /* 7 * n_frames */
} fdtd_keyframe_track;

typedef struct {
    int32_t shape;
    int32_t accel_kind;
    int32_t motion;
    int32_t mesh;         /* FDTD_SHAPE_MESH: index into fdtd_scene_desc.meshes; else 0 */
    double center[3];     /* body centre at t = 0 (world); a mesh's object-frame origin */
    double rotation[9];   /* row-major object->world rotation (identity if unused)    */
    double size[3];       /* sphere: size[0]=radius; box: half extents; ellipsoid: semi-axes */
    double accel_amplitude;
    double accel_t0;
    double accel_tau;
    double accel_dir[3];
    double velocity[3];   /* ballistic: x(t) = c + v t + g t^2 / 2                    */
    double gravity[3];
} fdtd_object_desc;

/* FDTD_PlaneConstraint (src/wavesolver/FDTD_PlaneConstraint.h:9-44) */
typedef struct {
    int32_t normal_dir;   /* 0,1,2 */
    int32_t normal_sign;  /* +1 / -1 */
    double height;
} fdtd_plane_desc;

/* GaussianPressureSource (src/wavesolver/GaussianPressureSource.h:11-51).  The
 * parser defaults (ImpulseResponseParser.cpp:657-669) are applied by
 * fdtd_gaussian_source_defaults(). */
typedef struct {
    double position[3];
    double width_time;
    double width_space;
    double offset_time;
    double normalize_constant;
} fdtd_gaussian_source_desc;

typedef struct {
    double cell_size;              /* <solver cellsize>                                   */
    int32_t divisions[3];          /* <solver_control_policy gridresolution> (per axis)   */
    int32_t boundary_condition_preset; /* 0 PML on every side; 1 walls +x, +z; 2 PML on +z only (MAC_Grid.cpp:4027-4101) */
    double domain_center[3];
    double sound_speed;
    double density;
    double time_step;              /* 1 / timestepfrequency                               */
    double pml_width;              /* cells                                               */
    double pml_strength;
    double air_viscosity_alpha;    /* MAC_Grid.cpp:926-930; 0: no viscosity              */
    double start_time;
    double end_time;               /* <= 0: no end                                         */
    int32_t n_objects;
    int32_t n_constraints;
    int32_t n_sources;
    int32_t n_listeners;
    const fdtd_object_desc* objects;
    const fdtd_plane_desc* constraints;
    const fdtd_gaussian_source_desc* sources;
    const double* listeners;       /* 3 * n_listeners, world coordinates                  */
    int32_t boundary_handling;     /* FDTD_BOUNDARY_* (<solver boundary_handling=>)       */
    int32_t n_meshes;
    const fdtd_mesh_desc* meshes;  /* meshes of the FDTD_SHAPE_MESH objects                */
    int32_t n_tracks;
    const fdtd_keyframe_track* tracks;  /* one per FDTD_MOTION_KEYFRAMED object          */
} fdtd_scene_desc;

enum {
    FDTD_BOUNDARY_RASTERIZE = 0,      /* ghost pressure from the neighbour and the wall acceleration */
    FDTD_BOUNDARY_FULLY_COUPLED = 1   /* image-point interpolation, all ghost cells solved together
                                         (spheres, boxes and meshes; fused kernels, single solves;
                                         moving bodies rebuild the rows on the host every step) */
};

enum {
    FDTD_PRECISION_FP64 = 0,              /* bit-faithful FP64 path                       */
    FDTD_PRECISION_FP32_COMPENSATED = 1   /* FP32 fields, increment-form accumulation     */
};

enum {
    FDTD_KERNEL_FUSED = 0,    /* region-split fused step: interior kernel + PML-shell kernel */
    FDTD_KERNEL_PHASED = 1    /* plain path: one kernel per reference phase (FP64 only)      */
};

typedef struct {
    int32_t precision;        /* FDTD_PRECISION_*                                        */
    int32_t device;           /* CUDA ordinal                                            */
    int32_t kernel;           /* FDTD_KERNEL_*                                           */
    int32_t graph_steps;      /* >0: capture this many steps per CUDA graph launch       */
    int32_t tile_y;           /* fused path: x planes a PML-shell thread marches over; 0: 8   */
    int32_t x_chunk;          /* fused path: interior x planes per thread (2, 4, 8); 0: 2        */
    int32_t pml_state;        /* FDTD_PML_STATE_*                                        */
    int32_t shell_staging;    /* FDTD_SHELL_STAGING_*                                    */
} fdtd_options;

enum {
    /* How the PML-shell kernel of FP32 solves on the reduced PML state stages its
     * loads (same results, bit for bit, either way):
     * RING: per-thread asynchronous copies (cp.async) into a shared-memory ring;
     * TMA: 3-D tensor copies (TMA) of every plane into a shared-memory ring, a
     * persistent producer / consumer kernel over tiles cut by absorbing axes,
     * for static single solves where the driver provides the tensor-map encoder
     * and the shell fits its windows (else RING);
     * AUTO: the faster of the two on B200 as measured, RING.
     * Batch members and moving scenes use RING. */
    FDTD_SHELL_STAGING_AUTO = 0,
    FDTD_SHELL_STAGING_RING = 1,
    FDTD_SHELL_STAGING_TMA = 2
};

enum {
    /* FP32 fused solves of static scenes with no solid cell inside the PML keep the
     * reduced PML state: along every axis without absorption at a PML cell the split
     * pressure and its two face velocities are replaced by one leapfrog increment
     * (exact in exact arithmetic; 8 instead of 14 words per slab cell and step).
     * Split-pressure and velocity fields cannot be read back then.  Every other
     * solve keeps the full state. */
    FDTD_PML_STATE_AUTO = 0,
    FDTD_PML_STATE_FULL = 1   /* always the reference's split pressures and face velocities */
};

typedef struct {
    int32_t divisions[3];
    int32_t n_listeners;
    int64_t n_cells;
    int64_t n_pml_cells;
    int64_t n_interior_cells;      /* non-PML cells                                     */
    int64_t device_bytes;          /* HBM held by this solver                           */
    int64_t step_index;
    double time;                   /* current simulation time                          */
    double time_step;
    double algorithmic_bytes_per_step; /* w*(3*N_interior + 14*N_pml)                  */
} fdtd_solver_info;

/* One ghost face, MAC_Grid::GhostCell (src/wavesolver/MAC_Grid.h:97-145). */
typedef struct {
    int32_t owner_cell;
    int32_t neighbour_cell;
    int32_t topology;        /* +-(dim+1), owner -> neighbour                       */
    int32_t type;            /* 0 object, 1 constraint                              */
    int32_t boundary_object; /* index into scene objects                            */
    int32_t _pad;
    uint64_t key;            /* Szudzik(min, max), MAC_Grid.h:108-116                */
} fdtd_ghost_face;

/* Per-cell classification byte returned by fdtd_solver_get_classification. */
enum {
    FDTD_CELL_BULK = 1,          /* _isBulkCell                                   */
    FDTD_CELL_GHOST = 2,         /* _isGhostCell                                  */
    FDTD_CELL_VALID_HISTORY = 4, /* _pressureCellHasValidHistory                  */
    FDTD_CELL_PML = 8,           /* _isPMLCell                                    */
    FDTD_CELL_CONSTRAINT = 16    /* solid because a plane constraint holds it      */
};

enum {
    FDTD_FIELD_PRESSURE = 0,        /* p^{n}   : _pCollocated[_pCollocatedInd]      */
    FDTD_FIELD_PRESSURE_PREV = 1,   /* p^{n-1}                                       */
    FDTD_FIELD_PML_PX = 2,          /* split pressures _p[0..2] (N cells)            */
    FDTD_FIELD_PML_PY = 3,
    FDTD_FIELD_PML_PZ = 4,
    FDTD_FIELD_VX = 5,              /* face velocities _v[0..2]                      */
    FDTD_FIELD_VY = 6,
    FDTD_FIELD_VZ = 7
};

/* One cell as MAC_Grid::GetCell fills a MAC_Grid::Cell (src/wavesolver/MAC_Grid.h:187-215,
 * MAC_Grid.cpp:4182-4258) for PML_WaveSolver::FetchCell (PML_WaveSolver.cpp:439-447).
 * The Cell's s_identity is r_identity spelt out ("Pressure Bulk / Solid / Ghost / PML
 * Cell") and its ghostCell pointer belongs to the finite-volume build; neither is here. */
typedef struct {
    int32_t index;            /* flat cell index (i*N1 + j)*N2 + k                            */
    int32_t indices[3];
    int32_t flags;            /* FDTD_CELL_* of the cell | FDTD_CELLINFO_*                   */
    int32_t n_gc_value;       /* gcValue.size(): 6 for a ghost cell outside the PML, else 0   */
    double r_identity;        /* PressureCellType (MAC_Grid.cpp:3977-3997): 0.5 bulk, 1 solid,
                                 -1 ghost, PML: -0.5 * max_d sigma_d(centre) / pml_strength */
    double centroid[3];
    double lower_corner[3];   /* centroid -/+ h/2                                             */
    double upper_corner[3];
    double gc_value[6];       /* ghost faces toward -x,+x,-y,+y,-z,+z: the face pressure the
                                 last step used (0 before the first step), -1 where that
                                 neighbour is not bulk; all -1 when n_gc_value is 0         */
    double p_directional[3];  /* split pressures _p[0..2]                                     */
    double p_full;            /* current pressure _pCollocated[_pCollocatedInd]                */
    double vx[2], vy[2], vz[2]; /* face velocities at the lower [0] and upper [1] face        */
    double h;
    double laplacian;         /* _pLaplacian[_pLaplacianInd], the Laplacian the last step kept
                                 (of the pressure two steps before p_full); see
                                 FDTD_CELLINFO_LAPLACIAN                                      */
} fdtd_cell;

enum {
    /* laplacian holds the reference's value: 0 before the first step; after it, solves
     * with air viscosity on the phased kernel (every cell) or on the fused kernels for
     * the non-PML cells of a static scene.  Otherwise it is NaN (the fused kernels keep
     * no Laplacian without air viscosity). */
    FDTD_CELLINFO_LAPLACIAN = 1 << 8,
    /* p_directional and the face velocities are held (NaN otherwise: the reduced PML
     * state, FDTD_PML_STATE_AUTO) */
    FDTD_CELLINFO_PML_STATE = 1 << 9
};

typedef struct fdtd_solver fdtd_solver;

/* ------------------------------------------------------------------------ */
/* library                                                                  */
int32_t fdtd_abi_version(void);
const char* fdtd_last_error(void);           /* thread-local message of the last failed call */
fdtd_status fdtd_device_count(int32_t* count);

/* Host-side failure injection for tests of the error paths (no counterpart in
 * the reference; nothing is done to the GPU): the (after+1)-th allocation of the
 * chosen kind from now on, counted over the process, fails as if memory were
 * exhausted, and the call that made it returns FDTD_ERR_OOM.  Device: the arena
 * of fdtd_solver_create (also reached by fdtd_batch_add and the solve server's
 * admissions).  Host: the pinned listener staging buffer of fdtd_solver_create
 * and the staging of fdtd_solver_get_field.  FDTD_INJECT_NONE disarms. */
enum { FDTD_INJECT_NONE = 0, FDTD_INJECT_DEVICE_ALLOC = 1, FDTD_INJECT_HOST_ALLOC = 2 };
fdtd_status fdtd_debug_inject_failure(int32_t what, int32_t after);

/* Parser defaults of <gaussian_pressure_source> (ImpulseResponseParser.cpp:657-669):
 * width_space <= 0 -> sound_speed*width_time; normalize_constant == 0 ->
 * 1/pow(sqrt(2*pi)*width_space, 3). */
fdtd_status fdtd_gaussian_source_defaults(fdtd_gaussian_source_desc* src, double sound_speed);

/* ------------------------------------------------------------------------ */
/* solver: replaces PML_WaveSolver                                          */

/* PML_WaveSolver(bbox, settings, objects) + Reinitialize_PML_WaveSolver(useBoundary=true, t0)
 * (PML_WaveSolver.cpp:78-146) + FDTD_AcousticSimulator::ResetStartTime (:458-523). */
fdtd_status fdtd_solver_create(const fdtd_scene_desc* scene, const fdtd_options* options,
                               fdtd_solver** out);
/* Releases the solver's streams and events; its device block is kept for the next
 * solver created on the same device (freed when an allocation would fail, when the
 * kept blocks pass 16 GiB or 256 blocks, oldest first, or by
 * fdtd_release_cached_memory). */
fdtd_status fdtd_solver_destroy(fdtd_solver* s);
/* Free the device blocks kept from destroyed solvers: of one device, or of all (device < 0). */
void fdtd_release_cached_memory(int32_t device);
/* Reinitialize_PML_WaveSolver(true, t0) + ResetCellHistory(true) (PML_WaveSolver.cpp:102-146) */
fdtd_status fdtd_solver_reset(fdtd_solver* s, double start_time);
/* n x (stepSystem() + FetchPressureData(listeners)) : SimWorld::StepWorld (SimWorld.cpp:507-592).
 * listener_out: host buffer of n_steps*n_listeners doubles (row = step), may be NULL.
 * Returns FDTD_END_OF_TIME when end_time was reached. */
fdtd_status fdtd_solver_step(fdtd_solver* s, int32_t n_steps, double* listener_out);
/* Same, with the listener series written to device memory (n_steps*n_listeners doubles)
 * and no host synchronisation. */
fdtd_status fdtd_solver_step_device(fdtd_solver* s, int32_t n_steps, void* device_listener_out);
/* FetchPressureData(listeningPoints, data, -1) at the current state (PML_WaveSolver.cpp:319-373) */
fdtd_status fdtd_solver_fetch_listeners(fdtd_solver* s, double* out);
fdtd_status fdtd_solver_info_get(fdtd_solver* s, fdtd_solver_info* info);
/* classifyCells_FAST result (MAC_Grid.cpp:3455-3891): flags_n (n_cells bytes, may be NULL);
 * faces (capacity *n_faces on entry, count on return; may be NULL to query the count). Faces are
 * ordered by (owner_cell, key). */
fdtd_status fdtd_solver_get_classification(fdtd_solver* s, uint8_t* flags_n, fdtd_ghost_face* faces,
                                           int64_t* n_faces);
/* Field read-back as doubles (FetchCell / GetGrid accessors). */
fdtd_status fdtd_solver_get_field(fdtd_solver* s, int32_t which, double* out, int64_t count);
/* The inverse of fdtd_solver_get_field (no counterpart in the reference): a dense
 * field into the solve (cells, or faces of one orientation, in the reference's flat
 * order).  FP32 FDTD_FIELD_PRESSURE_PREV sets the compensated increment from the
 * current pressure, so set FDTD_FIELD_PRESSURE first.  Split pressures and
 * velocities need the full PML state (FDTD_ERR_UNSUPPORTED on the reduced one). */
fdtd_status fdtd_solver_set_field(fdtd_solver* s, int32_t which, const double* in, int64_t count);
/* PML_WaveSolver::GetSolverDomain / GetSolverBBox (PML_WaveSolver.cpp:458-471): the
 * pressure grid's bounding box, min_bound + h * divisions = max_bound. */
fdtd_status fdtd_solver_domain(fdtd_solver* s, double min_bound[3], double max_bound[3]);
/* PML_WaveSolver::FetchCell (PML_WaveSolver.cpp:439-447): cell cell_index (flat, in
 * [0, n_cells)) at the current state. */
fdtd_status fdtd_solver_fetch_cell(fdtd_solver* s, int64_t cell_index, fdtd_cell* out);
/* PML_WaveSolver::SampleAxisAlignedSlice -> MAC_Grid::SampleAxisAlignedSlice
 * (PML_WaveSolver.cpp:449-458, MAC_Grid.cpp:1941-1963): the cells of plane
 * k = min((int)((offset - (bmin[dim] - h/2)) / h), N[dim] - 1) across axis dim, i over
 * N[(dim+1)%3] outer, j over N[(dim+2)%3] inner.  *count <- N[(dim+1)%3]*N[(dim+2)%3];
 * out may be NULL to query it, else capacity must reach it.  An offset a cell or more
 * below the grid (k < 0) is FDTD_ERR_INVALID_ARG. */
fdtd_status fdtd_solver_sample_slice(fdtd_solver* s, int32_t dim, double offset, fdtd_cell* out,
                                     int64_t capacity, int64_t* count);
/* Synchronise the solver's stream. */
fdtd_status fdtd_solver_synchronize(fdtd_solver* s);
/* The cudaStream_t every kernel of this solver is launched on (for event timing). */
void* fdtd_solver_stream(fdtd_solver* s);
const char* fdtd_solver_last_error(fdtd_solver* s);
/* Capture now the CUDA graph that the next graph_steps-long chunk of
 * fdtd_solver_step* would capture on its first use (no counterpart in the
 * reference): nothing runs on the GPU, so timed stepping afterwards pays no
 * capture cost.  A no-op without graph_steps, for moving scenes and before
 * the first (classifying) step. */
fdtd_status fdtd_solver_prepare_graphs(fdtd_solver* s);
/* ------------------------------------------------------------------------ */
/* output files (fdtd_io.cpp)                                               */

/* IO::writeMatrixX<double>(..., IO::BINARY) (src/utils/IO/IO.h:107-160) and
 * MATRIX::write (src/linearalgebra/MATRIX_FAST.cpp:134-155): int32 rows, int32
 * cols, rows*cols doubles, row-major. */
fdtd_status fdtd_matrix_write(const char* path, int32_t rows, int32_t cols, const double* data);
/* the reader (MATRIX::read, MATRIX_FAST.cpp:160-187); data may be NULL to query the size */
fdtd_status fdtd_matrix_read(const char* path, int32_t* rows, int32_t* cols, double* data, int64_t capacity);
/* FDTD_AcousticSimulator::_SaveSimulationSnapshot (FDTD_AcousticSimulator.cpp:381-415):
 * snapshot_<numbering>_{p_pml_d, v_pml_d, p_collocated_d, p_pml_full, p_collocated_ind}
 * composed with the output pattern's %s (CompositeFilename, :109-125; NULL: "%s").
 * The collocated buffer the next step overwrites unread is written as zeros.
 * Needs the full PML state. */
fdtd_status fdtd_solver_save_snapshot(fdtd_solver* s, const char* output_pattern, const char* numbering);
/* The inverse (no counterpart in the reference): pressures, split pressures and
 * velocities of a snapshot of a grid of the same size into this solve. */
fdtd_status fdtd_solver_load_snapshot(fdtd_solver* s, const char* output_pattern, const char* numbering);
/* SaveSolverConfig's position files (FDTD_AcousticSimulator.cpp:146-230, :647-661):
 * pressure_vertex_position.dat, velocity_<d>_vertex_position.dat, listening_position.dat */
fdtd_status fdtd_solver_save_config(fdtd_solver* s, const char* output_pattern);
/* _SavePressureTimestep / _SaveVelocityTimestep (FDTD_AcousticSimulator.cpp:253-307):
 * which = FDTD_FIELD_PRESSURE or FDTD_FIELD_V{X,Y,Z}, x-fastest (n x 1) matrix */
fdtd_status fdtd_solver_save_field_timestep(fdtd_solver* s, int32_t which, const char* path);

/* FULLY_COUPLED diagnostics (no counterpart in the reference; it prints the same
 * figures every step, MAC_Grid.cpp:1413-1418): ghost-face rows, rows interpolated
 * at the image point, rows that fell back to the rasterized value, and the
 * BiCGSTAB iterations of the last step (negative: not converged). */
fdtd_status fdtd_solver_boundary_info(fdtd_solver* s, int64_t* n_rows, int64_t* n_immersed, int64_t* n_fallback,
                                      int32_t* last_iterations);
/* PML state in effect: FDTD_PML_STATE_FULL, or FDTD_PML_STATE_AUTO when the
 * reduced state is used (no counterpart in the reference). */
int32_t fdtd_solver_pml_state(fdtd_solver* s);
/* Staging of the reduced-state PML-shell kernel in effect: FDTD_SHELL_STAGING_TMA
 * or FDTD_SHELL_STAGING_RING; -1 when the solve keeps the full PML state (no
 * counterpart in the reference). */
int32_t fdtd_solver_shell_staging(fdtd_solver* s);
/* Kernel launches issued by the most recent fdtd_solver_step* call. */
int64_t fdtd_solver_last_launch_count(fdtd_solver* s);
/* Steps since creation whose PML-shell kernel ran beside the step's cell
 * classification (moving bodies two cells clear of the PML); the others ran it
 * after.  Execution statistics only: the results are the same either way. */
int64_t fdtd_solver_overlapped_steps(fdtd_solver* s);
/* Bytes this handle has copied from host to device memory and back since its
 * creation (scene tables, meshes, per-step object poses, listener rows, status
 * words); no counterpart in the reference, whose state lives in host memory. */
fdtd_status fdtd_solver_transfer_bytes(fdtd_solver* s, int64_t* host_to_device, int64_t* device_to_host);

/* Profiling hook (no counterpart in the reference): the step kernels n_launches
 * times back to back (alternating buffer parity, no prologue, source or listener
 * work), captured into a CUDA graph that is replayed once untimed and once
 * between two CUDA events on the solver stream: device time only, whatever the
 * host's launch rate.  Returns the elapsed milliseconds of the timed replay.  The
 * fields are left in an unspecified state; use a solver created for measurement. */
fdtd_status fdtd_solver_time_stencil(fdtd_solver* s, int32_t n_launches, float* elapsed_ms);
/* The same for one part of the step: which = 0 the step kernels (as
 * fdtd_solver_time_stencil),
 * 1 the interior kernel, 2 the PML-shell kernel, 3 the ghost-cell list kernel,
 * 4 the listener kernel.  Parts 1-4 need FDTD_KERNEL_FUSED.  The fields are
 * left in an unspecified state (timing only). */
fdtd_status fdtd_solver_time_kernel(fdtd_solver* s, int32_t which, int32_t n_launches, float* elapsed_ms);

/* Interior leapfrog step that allocates nothing.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc where they step
 * the field — real-time callbacks that must not block on the allocator or on
 * the synchronisation an allocation may imply, and hosts whose own memory pool
 * already holds the GPU's free memory.
 * One step of the plain path's Laplacian + leapfrog (MAC_Grid.cpp:187-299,
 * :921-935) on the box lo <= (i,j,k) < hi of a dims[0] x dims[1] x dims[2] FP64
 * grid (flat index i*dims[1]*dims[2] + j*dims[2] + k, device pointers), every box
 * cell treated as a bulk, non-PML cell with no solid neighbour:
 *   p_next = 2 p_curr - p_prev + c2k2 * lap_scale * sum_d (p_+ + p_- - 2 p_curr)
 * p_next may equal p_prev (in place); cells outside the box are not written.
 * Requires 1 <= lo < hi <= dims-1 per axis and at most FDTD_NOALLOC_MAX_CELLS
 * box cells (FDTD_ERR_INVALID_ARG otherwise).  The Laplacian scratch is one
 * static device array of FDTD_NOALLOC_MAX_CELLS doubles (8 MiB) that every GPU
 * loading the library keeps until exit.  The first call on a device (and the
 * first after a device reset gave it a new context) looks up that array's
 * device address (cudaGetSymbolAddress) with the device current; make that
 * first call before any stream capture.  Calls share the array, so calls that
 * overlap on the GPU race; serialise them on one stream.  `stream` is a
 * cudaStream_t (NULL: the legacy default stream); the call only enqueues work. */
#define FDTD_NOALLOC_MAX_CELLS (1 << 20)
fdtd_status fdtd_interior_step_noalloc(const double* p_curr, const double* p_prev, double* p_next,
                                       const int32_t dims[3], const int32_t lo[3], const int32_t hi[3],
                                       double c2k2, double lap_scale, void* stream);

/* Snapshot / restore of the resident state (_SaveSimulationSnapshot,
 * FDTD_AcousticSimulator.cpp:381-415).  bytes: query with buffer NULL. */
fdtd_status fdtd_solver_snapshot(fdtd_solver* s, void* buffer, int64_t* bytes);
fdtd_status fdtd_solver_restore(fdtd_solver* s, const void* buffer, int64_t bytes);

/* ------------------------------------------------------------------------ */
/* Batches of independent static solves stepped together.  No counterpart in
 * the reference, which steps its sim units one after the other
 * (SimWorld.cpp:517-590); each member produces exactly what an fdtd_solver of
 * the same scene and options produces.  Per step the whole batch costs a fixed
 * number of kernel launches; members may have different grids, step counts,
 * objects, sources and listeners, and retire when their steps are done. */
typedef struct fdtd_batch fdtd_batch;
fdtd_status fdtd_batch_create(int32_t n, const fdtd_scene_desc* scenes, const int32_t* steps,
                              const fdtd_options* options, fdtd_batch** out);
/* add a member (its first, classifying step runs at once); returns its index,
 * which may be the index of a released member */
fdtd_status fdtd_batch_add(fdtd_batch* b, const fdtd_scene_desc* scene, int32_t steps, int32_t* member);
/* advance every active member by up to n_steps; *n_active: members still running */
fdtd_status fdtd_batch_step(fdtd_batch* b, int32_t n_steps, int32_t* n_active);
/* run until every member has finished */
fdtd_status fdtd_batch_run(fdtd_batch* b);
fdtd_status fdtd_batch_member_info(fdtd_batch* b, int32_t member, int64_t* steps_done, int64_t* steps_total,
                                   int32_t* n_listeners, int32_t* status);
/* listener series of a member so far: steps_done x n_listeners doubles */
fdtd_status fdtd_batch_output(fdtd_batch* b, int32_t member, double* out, int64_t count);
/* The state of a member (fdtd_solver_snapshot of its solve; query the size with
 * buffer NULL).  With fdtd_batch_add_snapshot it moves a member out of device
 * memory and back, as the solve server's eviction does. */
fdtd_status fdtd_batch_member_snapshot(fdtd_batch* b, int32_t member, void* buffer, int64_t* bytes);
/* Add a member that continues from a snapshot of a member (or solver) of the
 * same scene and options: steps_total counts from the solve's start, rows holds
 * its listener series so far (steps_done x n_listeners doubles, steps_done = the
 * snapshot's step; NULL when n_listeners is 0).  No step runs here. */
fdtd_status fdtd_batch_add_snapshot(fdtd_batch* b, const fdtd_scene_desc* scene, int32_t steps_total,
                                    const void* snapshot, int64_t bytes, const double* rows, int64_t steps_done,
                                    int32_t* member);
/* stop a member if it still runs, free its device memory and series; its index becomes free */
fdtd_status fdtd_batch_release(fdtd_batch* b, int32_t member);
fdtd_status fdtd_batch_destroy(fdtd_batch* b);
void* fdtd_batch_stream(fdtd_batch* b);
int64_t fdtd_batch_last_launch_count(fdtd_batch* b);
int64_t fdtd_batch_device_bytes(fdtd_batch* b);
/* Device bytes of the arena a solver of this scene and options allocates (admission by
 * HBM footprint); -1 when the scene is invalid. */
int64_t fdtd_scene_device_bytes(const fdtd_scene_desc* scene, const fdtd_options* options);
/* The fdtd_solver_info a solver of this scene would report at creation (grid,
 * PML / interior cell counts, device and algorithmic bytes), computed on the
 * host without a device. */
fdtd_status fdtd_scene_info(const fdtd_scene_desc* scene, const fdtd_options* options, fdtd_solver_info* info);

/* ------------------------------------------------------------------------ */
/* Solve server: continuous batching of submitted scenes.  No counterpart in the
 * reference.  A worker thread owns one fdtd_batch; between chunks of batched
 * steps it admits queued requests in arrival order while their device bytes
 * (fdtd_scene_device_bytes) fit the budget and a member slot is free, and
 * retires finished ones, whose series stay on the host until collected.  A
 * request's series equals that of an fdtd_solver of the same scene and
 * options, whatever else runs beside it. */
typedef struct fdtd_server fdtd_server;

typedef struct {
    int64_t hbm_budget_bytes;  /* device bytes the members may hold; 0: 90% of free memory at create */
    int32_t max_members;       /* members stepped together; 0: 256; 1 gives FIFO service           */
    int32_t chunk_steps;       /* batched steps between admissions; 0: max(graph_steps, 32)       */
    int32_t preempt;           /* 1: evict running members to admit a shorter queue head (below)   */
} fdtd_server_config;
/* Eviction (preempt = 1; the reference's snapshot, FDTD_AcousticSimulator.cpp:381-415,
 * used as the server's preemption): when the request at the head of the queue
 * does not fit the free budget, running members with more than twice its
 * cell-steps still to go are evicted, most remaining work first, until it fits.
 * An evicted member's state (fdtd_batch_member_snapshot) and listener rows stay
 * in host memory, its device memory is released, and it goes back into the
 * queue right behind the head; re-admitted, it continues where it stopped and
 * its series equals an uninterrupted solve's bit for bit. */

enum { FDTD_REQ_QUEUED = 0, FDTD_REQ_RUNNING = 1, FDTD_REQ_DONE = 2, FDTD_REQ_FAILED = 3,
       FDTD_REQ_CANCELLED = 4 };

typedef struct {
    int64_t submitted, completed, failed, queued, running;
    int64_t peak_members;
    int64_t peak_device_bytes;      /* sum of admitted footprints                               */
    double p50_latency_s, p99_latency_s, mean_latency_s;  /* submit -> done, completed requests */
    double span_s;                  /* first submit -> last completion                         */
    double solves_per_s;            /* completed / span_s                                      */
    double cell_steps_per_s;        /* sum of cells x steps of completed requests / span_s     */
    int64_t device_bytes_in_use;    /* footprints of the members now admitted                  */
    int64_t cancelled;              /* requests cancelled                                      */
    int64_t evictions;              /* members evicted to host memory (preempt)                */
} fdtd_server_stats;

fdtd_status fdtd_server_create(const fdtd_options* options, const fdtd_server_config* config, fdtd_server** out);
/* queue a copy of the scene for `steps` steps; FDTD_ERR_INVALID_ARG for an invalid scene or
 * one whose footprint exceeds the budget */
fdtd_status fdtd_server_submit(fdtd_server* srv, const fdtd_scene_desc* scene, int32_t steps, int64_t* request);
/* state (FDTD_REQ_*), steps done, and for failed requests the status */
fdtd_status fdtd_server_poll(fdtd_server* srv, int64_t request, int32_t* state, int64_t* steps_done,
                             int32_t* status);
/* block until the request is done or failed; FDTD_ERR_TIMEOUT after timeout_s (< 0: no limit) */
fdtd_status fdtd_server_wait(fdtd_server* srv, int64_t request, double timeout_s);
/* steps x n_listeners doubles and the latency; the request is forgotten afterwards */
fdtd_status fdtd_server_result(fdtd_server* srv, int64_t request, double* out, int64_t count, int64_t* steps,
                               int32_t* n_listeners, double* latency_s);
/* block until every submitted request is done, failed or cancelled */
fdtd_status fdtd_server_drain(fdtd_server* srv, double timeout_s);
/* Cancel a queued or running request: a queued one leaves the queue, a running
 * one is stopped at the end of the batched chunk in progress and its device
 * memory released; its state becomes FDTD_REQ_CANCELLED and fdtd_server_wait /
 * fdtd_server_result return FDTD_ERR_CANCELLED.  FDTD_ERR_INVALID_ARG for an
 * unknown or already finished request.  (No counterpart in the reference.) */
fdtd_status fdtd_server_cancel(fdtd_server* srv, int64_t request);
fdtd_status fdtd_server_stats_get(fdtd_server* srv, fdtd_server_stats* stats);
/* the error text of a failed request */
const char* fdtd_server_request_error(fdtd_server* srv, int64_t request);
fdtd_status fdtd_server_destroy(fdtd_server* srv);

/* ------------------------------------------------------------------------ */
/* XML scene reader (ImpulseResponseParser subset, ImpulseResponseParser.cpp:55-751) */
typedef struct fdtd_scene fdtd_scene;
fdtd_status fdtd_scene_from_xml(const char* path, fdtd_scene** out);
const fdtd_scene_desc* fdtd_scene_desc_get(const fdtd_scene* sc);
/* int steps from <number_of_timesteps> (0 if absent) and the output pattern */
int32_t fdtd_scene_number_of_steps(const fdtd_scene* sc);
const char* fdtd_scene_output_pattern(const fdtd_scene* sc);
void fdtd_scene_free(fdtd_scene* sc);

/* A kinematics file of FDTD_RigidObject_Blender_Animator::ReadObjectKinData
 * (FDTD_RigidObject_Animator.cpp:79-122): one line per frame, "frame tx ty tz qw
 * qx qy qz"; w is clamped to [-1, 1] and every rotation is turned by -90 degrees
 * about x (Blender's z-up to y-up, as the reference's animator does).  frames:
 * 7 * n_frames doubles as in fdtd_keyframe_track (NULL to query n_frames). */
fdtd_status fdtd_read_kinematics(const char* path, int32_t* n_frames, double* frames, int64_t capacity);
/* Pose of a keyframed object at time t (host query, no GPU): centre com[3] and
 * the rotation R[9] (row-major) that turns the rest pose. */
fdtd_status fdtd_keyframe_pose(const fdtd_keyframe_track* track, double t, double* com, double* rotation);

/* Wavefront .obj surface mesh (MeshObjReader::read with a scale, as the
 * <rigid_object scale=> attribute applies it): the "v" and "f" records, polygons
 * fanned into triangles, indices made 0-based.  Call with NULL arrays for the
 * counts, then with arrays of 3 * count entries. */
fdtd_status fdtd_read_obj(const char* path, double scale, int32_t* n_vertices, int32_t* n_triangles,
                          double* vertices, int32_t* triangles);

/* Signed distance (negative inside) of n points to a closed mesh, in the mesh's
 * frame: the query the cell classification makes of mesh bodies (exact distance
 * to the closest triangle point, sign of the closest feature's pseudo-normal),
 * on the host.  FDTD_ERR_GEOMETRY for a mesh that is open or inconsistently
 * oriented. */
fdtd_status fdtd_mesh_signed_distance(const fdtd_mesh_desc* mesh, int64_t n, const double* points, double* out);

/* all_audio.dat writer (AudioOutput, src/wavesolver/AudioOutput.cpp:27-64): appends
 * n_steps*n_listeners raw doubles. */
fdtd_status fdtd_audio_append(const char* path, const double* data, int64_t count);

#ifdef __cplusplus
}
#endif
#endif /* FDTD_C_H */
