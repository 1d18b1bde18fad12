/* ag2d — B200-native collision and contact pipeline for the PS_AGONY2D world/body/shape/step API.
 *
 * C ABI of libag2d.so: opaque handles, plain pointers and sizes, int32 status codes. Every entry point below
 * names the reference interface it replaces (paths relative to PhysicsSimulation-Agony/PS_AGONY2D/ in
 * Shadow001111/PhysicsSimulation-Agony). The reference is statically linked C++ with no FFI of its own; these are
 * the calls its Simulation / ObjectAPI boundary maps onto.
 *
 * Threading: a world is driven by one host thread at a time (the reference's Simulation is single-caller too,
 * Simulation.h:36). Distinct worlds and batches may be driven from distinct threads.
 * Errors: functions return AG2D_OK or a negative AG2D_ERR_*; ag2d_last_error_string() describes the last failure
 * on the calling thread. Nothing aborts the process (the reference aborts or returns std::nullopt).
 */
#ifndef AG2D_H
#define AG2D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AG2D_OK 0
#define AG2D_ERR_INVALID_ARG (-1)
#define AG2D_ERR_OOM (-2)
#define AG2D_ERR_CAPACITY (-3)   /* a buffer overflowed and could not be regrown */
#define AG2D_ERR_TIMEOUT (-4)    /* a bounded device-side wait gave up (status word set, GPU left usable) */
#define AG2D_ERR_CUDA (-5)
#define AG2D_ERR_NO_DEVICE (-6)
#define AG2D_ERR_UNSUPPORTED (-7)

typedef struct ag2d_world ag2d_world;
typedef struct ag2d_batch ag2d_batch;

/* Mirrors Simulation::SimulationSettings (Simulation.h:50-76), FixedClock::Settings (SimulationImpl/FixedClock.h:
 * 12-17) and Integrator::Settings (Integration/Integrator.h:14-19). */
typedef struct ag2d_world_settings {
    float dt;                        /* fixed step (clockSettings.updateInterval) */
    uint32_t velocity_iterations;    /* collisionVelocitySolvingIterations */
    uint32_t position_iterations;    /* collisionPositionSolvingIterations */
    float gravity_x, gravity_y;      /* integratorSettings.gravity */
    float angular_damping;           /* integratorSettings.angularVelocityDamping (1 = off) */
    float sleep_speed;               /* sleepSpeedThreshold */
    float sleep_time;                /* sleepTimeThreshold */
    int32_t ccd;                     /* continuousCollisionEnabled */
    int32_t device;                  /* CUDA device ordinal */
} ag2d_world_settings;

/* Mirrors BodyCreateParams (SimulationImpl/ObjectCreateParams.h:14-24). mass 0 makes a static body. */
typedef struct ag2d_body_desc {
    float x, y, rotation;
    float vx, vy, angular_velocity;
    float mass;
    uint32_t material;
} ag2d_body_desc;

/* Per-step counters (the step statistics the reference keeps in its DebugData). */
typedef struct ag2d_counters {
    uint32_t status;        /* device status bits of the last step */
    uint32_t pairs;         /* broad-phase candidate pairs */
    uint32_t manifolds;     /* contact manifolds */
    uint32_t colors;        /* solver colours */
    uint32_t woke;          /* bodies woken */
    uint32_t slept;         /* bodies put to sleep */
    uint32_t warm_hits;     /* manifolds warm-started */
    uint32_t sleeping;      /* bodies sleeping after the step */
    uint32_t ccd_hits;      /* bodies moved back by continuous collision detection in the last step */
    uint32_t restored;      /* manifolds of woken islands that joined the last step whole (from the sleep store) */
    uint32_t events;        /* collision events recorded in the last step */
    uint32_t stored;        /* sleeping-island manifolds held when the last step began */
    uint64_t steps;         /* steps taken by this world */
    uint64_t launches;      /* kernel launches issued by this world so far */
    uint64_t list_rebuilds; /* work-list rebuilds after sleep/wake changes */
    uint64_t retries;       /* steps re-run after a buffer overflow (state restored, buffers grown) */
    uint64_t regrows;       /* capacity growths */
    double host_ms;         /* host wall time spent inside ag2d_world_step so far */
    double sync_ms;         /* of which waiting for the device at the end of steps */
    uint64_t device_allocs; /* device buffer allocations made by the library in this process so far (each one
                               synchronises the device; a steady run of steps makes none) */
} ag2d_counters;

/* Phases timed by ag2d_world_phase_times (index into the returned array). */
enum ag2d_timed_phase {
    AG2D_T_INTEGRATE = 0, AG2D_T_POSE, AG2D_T_TREE_DYNAMIC, AG2D_T_TREE_OTHER, AG2D_T_QUERY, AG2D_T_NARROW,
    AG2D_T_COMPACT, AG2D_T_WARM, AG2D_T_WAKE, AG2D_T_COLOR, AG2D_T_SOLVE, AG2D_T_ISLANDS, AG2D_T_SORT,
    AG2D_T_LBVH, AG2D_T_CCD, AG2D_T_COUNT
};

/* Launch shapes chosen by ag2d_world_autotune. */
typedef struct ag2d_tuning {
    uint32_t team_colliders;   /* batched solver: colliders per CTA team of consecutive worlds (0: single world) */
    uint32_t team_threads;     /* batched solver: threads per team CTA (0: single world) */
    uint32_t query_threads;    /* pair-query block size */
    uint32_t narrow_threads;   /* narrow-phase block size */
    float solve_ms, query_ms, narrow_ms;   /* device time per step of each phase at the chosen setting */
    uint32_t team_cons_on_chip;  /* batched solver: a team's constraint records kept in shared memory (1) or not */
    uint32_t big_team_mode;      /* batched solver, worlds larger than a team: bit 0 = 256-thread CTAs (else 512),
                                    bit 1 = record loads pipelined one phase ahead */
} ag2d_tuning;

/* Reference-layout world state for ag2d_world_load_state: every array in the reference's dense order, as its
 * SoA viewers expose them (SoA/BodySoA.h:14-36, SoA/ColliderSoA.h:10-32, SoA/Shapes/*.h). Group starts are
 * GroupRanges::starts (GroupRanges.h:130-157): static, sleeping, dynamic, end. */
typedef struct ag2d_state_desc {
    uint32_t n_bodies, n_colliders, n_circles, n_boxes, n_polygons, n_materials;
    const uint32_t* body_group_starts;   /* [4] */
    const float *com_x, *com_y, *vel_x, *vel_y, *rotation, *angular_velocity;
    const float *inv_mass, *inv_inertia, *rot_cos, *rot_sin, *wrap_count, *bound_radius, *sleep_timer;
    const uint32_t* sleep_island;        /* may be NULL */
    const uint32_t *col_body, *col_shape_type, *col_shape_index, *col_material;
    const float *col_com_offset_x, *col_com_offset_y, *col_local_rotation;
    const float* circle_radius;          /* [n_circles] */
    const float *box_half_width, *box_half_height;   /* [n_boxes] */
    const uint32_t* poly_count;          /* [n_polygons] vertex counts */
    const float* poly_vertices;          /* xy pairs, concatenated */
    const float* poly_normals;           /* xy pairs, concatenated */
    const float* materials;              /* [n_materials][3]: elasticity, static friction, dynamic friction */
    /* Optional (NULL: computed by the next spatial pass): each collider's world pose and AABB as the state holds
     * them (ColliderSoA worldPos / worldRotationCos / Sin, aabbMin / Max). */
    const float *col_world_x, *col_world_y, *col_world_cos, *col_world_sin;
    const float *col_aabb_min_x, *col_aabb_min_y, *col_aabb_max_x, *col_aabb_max_y;
    /* Capsules (CapsuleSoA): colliders of shape type 3 index these arrays. */
    uint32_t n_capsules;
    const float *capsule_half_length, *capsule_radius;   /* [n_capsules] */
} ag2d_state_desc;

/* Readable / writable world fields (ag2d_world_read / ag2d_world_write). Body and collider arrays are float32 or
 * uint32 in dense order; pair arrays are uint32 pairs; manifolds are 64-byte records (ag2d_manifold). */
enum ag2d_field {
    AG2D_BODY_COM_X = 1, AG2D_BODY_COM_Y, AG2D_BODY_VEL_X, AG2D_BODY_VEL_Y, AG2D_BODY_ROTATION,
    AG2D_BODY_ANGULAR_VELOCITY, AG2D_BODY_ROT_COS, AG2D_BODY_ROT_SIN, AG2D_BODY_WRAP_COUNT, AG2D_BODY_SLEEP_TIMER,
    AG2D_BODY_STATE /* uint32: 0 static, 1 sleeping, 2 dynamic */, AG2D_BODY_SLEEP_ISLAND,
    AG2D_BODY_POSE /* float32 x, y, rotation per body: one read of the pose array (a renderer's frame) */,
    AG2D_BODY_INV_MASS, AG2D_BODY_INV_INERTIA,
    AG2D_COL_WORLD_X = 32, AG2D_COL_WORLD_Y, AG2D_COL_WORLD_ROTATION, AG2D_COL_WORLD_COS, AG2D_COL_WORLD_SIN,
    AG2D_COL_AABB_MIN_X, AG2D_COL_AABB_MIN_Y, AG2D_COL_AABB_MAX_X, AG2D_COL_AABB_MAX_Y,
    AG2D_COL_BODY /* uint32: the owner body's dense index (read only) */,
    AG2D_DYN_SORTED = 64,   /* dynamic tree: collider indices in Morton order */
    AG2D_DYN_MORTON,        /* dynamic tree: sorted Morton keys */
    AG2D_PAIRS,             /* candidate pairs (uint32 a, b) */
    AG2D_MANIFOLDS,         /* current manifolds */
    AG2D_PREV_MANIFOLDS,    /* previous step's manifolds (warm-start source) */
    AG2D_SOLVE_ORDER,       /* uint32 manifold index per solving slot (colour-major) */
    AG2D_COLOR_STARTS,      /* uint32 [colors + 1] */
    AG2D_ISLAND_MANIFOLDS,  /* manifolds of sleeping islands, kept until their island wakes (world-grouped) */
    AG2D_ISLAND_IDS,        /* uint32 island of each stored manifold: the dense index of the island's root body
                               (writable after AG2D_ISLAND_MANIFOLDS, with the same count) */
};

/* Manifold record (NarrowPhaseCollisionDetector.h:26-61 with dense collider indices instead of handles). */
typedef struct ag2d_manifold {
    uint32_t a, b;
    float nx, ny, depth;
    uint32_t count, id0, id1;
    float px0, py0, px1, py1;
    float jn0, jt0, jn1, jt1;
} ag2d_manifold;

/* Debug phases (ag2d_world_run_phase): one phase of the step on the current state, for parity checks. */
enum ag2d_phase {
    AG2D_PHASE_INTEGRATE = 1,      /* integrate + wrap + rotation cos/sin over dynamic bodies */
    AG2D_PHASE_SPATIAL_FULL,       /* collider poses + AABBs over all colliders */
    AG2D_PHASE_SPATIAL_DYNAMIC,    /* collider poses + AABBs over dynamic colliders */
    AG2D_PHASE_BROAD,              /* bounds, Morton, sort, LBVH, pair query */
    AG2D_PHASE_NARROW,             /* narrow phase on AG2D_PAIRS, warm start from AG2D_PREV_MANIFOLDS */
    AG2D_PHASE_SOLVE,              /* colouring + solver on AG2D_MANIFOLDS */
    AG2D_PHASE_ISLANDS,            /* islands + sleep flags from AG2D_MANIFOLDS */
    AG2D_PHASE_COLLIDE,            /* collision detection alone: dynamic poses + AABBs, broad, narrow (no warm start) */
    AG2D_PHASE_CCD,                /* continuous collision: sweep fast dynamic colliders against static ones, move
                                      hit bodies back (uses the poses AG2D_PHASE_INTEGRATE recorded) */
    AG2D_PHASE_WAKE,               /* wake the sleeping islands AG2D_MANIFOLDS touch, then bring their stored
                                      manifolds into AG2D_MANIFOLDS (Simulation.cpp:440-444) */
    AG2D_PHASE_EVENTS              /* collision events of AG2D_MANIFOLDS from the current velocities (the solver's
                                      input), into ag2d_world_collision_events; no callback is called */
};

/* ---- library ---- */
const char* ag2d_last_error_string(void);
int32_t ag2d_version(void);
int32_t ag2d_device_count(int32_t* out_count);

/* ---- world lifecycle: Simulation::Simulation / ~Simulation (Simulation.cpp:21-30) ---- */
int32_t ag2d_world_create(const ag2d_world_settings* settings, ag2d_world** out_world);
int32_t ag2d_world_destroy(ag2d_world* world);

/* Simulation::createMaterial (Simulation.cpp:76-79; values clamped like MaterialManager::sanitize,
 * SimulationImpl/MaterialManager.h:29-35). Index 0 is the default material (elasticity 1, no friction). */
int32_t ag2d_world_add_material(ag2d_world* world, float elasticity, float static_friction, float dynamic_friction,
                                uint32_t* out_index);

/* ObjectAPI::createCircleH / createBoxH / createPolygonH (SimulationAPIs/ObjectAPI.h:61-65;
 * ObjectManager::createCircle/createBox/createPolygon, SimulationImpl/ObjectManager.cpp:233-349). Mass, inertia,
 * centre of mass and polygon recentring follow the reference's PhysicsGeometry. Polygons must be convex after
 * outline cleaning, concave outlines split into convex pieces, one collider each. The handle is
 * (generation << 32) | slot and stays valid across other creations. */
int32_t ag2d_world_add_circle(ag2d_world* world, const ag2d_body_desc* body, float radius, uint64_t* out_handle);
int32_t ag2d_world_add_box(ag2d_world* world, const ag2d_body_desc* body, float width, float height,
                           uint64_t* out_handle);
int32_t ag2d_world_add_polygon(ag2d_world* world, const ag2d_body_desc* body, const float* vertices_xy,
                               uint32_t vertex_count, uint64_t* out_handle);
/* ObjectAPI::createBodyH (ObjectAPI.h:61; ObjectManager::createBody, ObjectManager.cpp:71-88): a body with the
 * descriptor's pose, velocities and mass, the given inertia and local centre of mass, and no collider yet. */
int32_t ag2d_world_create_body(ag2d_world* world, const ag2d_body_desc* body, float inertia, float com_x,
                               float com_y, uint64_t* out_handle);
/* ObjectAPI::create{Circle,Box,Polygon,Capsule}Collider (ObjectAPI.h:29-32; ObjectManager.cpp:90-231): a collider
 * on an existing body at a local offset and rotation. shape: 0 circle (params[0] radius), 1 box (params = width,
 * height), 2 polygon (xy / n_vertices: a convex outline, recentred on its centroid with the shift added to the
 * offset; a concave outline becomes one collider per convex piece, the first returned), 3 capsule (params =
 * length, radius). The body's mass and inertia stay as created. out_collider: the collider's dense index. */
int32_t ag2d_world_add_collider(ag2d_world* world, uint64_t body, int32_t shape, float local_x, float local_y,
                                float local_rotation, uint32_t material, const float* params, const float* xy,
                                uint32_t n_vertices, uint32_t* out_collider);
/* ObjectAPI::createCapsuleH (SimulationAPIs/ObjectAPI.h:65; ObjectManager::createCapsule, ObjectManager.cpp:351-388):
 * a capsule body whose core of 'length' (cap centre to cap centre) lies along the body's x axis, swept by 'radius'. */
int32_t ag2d_world_add_capsule(ag2d_world* world, const ag2d_body_desc* body, float length, float radius,
                               uint64_t* out_handle);
/* Creates 'count' bodies in one call: the same bodies, in the same order, as the matching add_circle / add_box /
 * add_polygon calls (a scene loader's loop over ObjectAPI::create*, ObjectAPI.h:20-45, without a call per body).
 * kinds[i]: 0 circle (params[2i] = radius), 1 box (params[2i], params[2i+1] = width, height), 2 polygon
 * (poly_counts[i] vertex pairs at poly_xy + 2 * poly_offsets[i]). out_handles may be NULL. Stops at the first body
 * that cannot be created (its index is in the error string); the bodies before it stay created. */
int32_t ag2d_world_add_bodies(ag2d_world* world, uint32_t count, const ag2d_body_desc* bodies,
                              const uint32_t* kinds, const float* params, const uint32_t* poly_offsets,
                              const uint32_t* poly_counts, const float* poly_xy, uint64_t* out_handles);
/* Dense body index of a handle (ObjectAPI::getBodyIndex, ObjectAPI.h:53), or UINT32_MAX if stale. */
uint32_t ag2d_world_body_index(ag2d_world* world, uint64_t handle);

/* ---- deferred body commands: ObjectAPI::destroyBody / setBody* (SimulationAPIs/ObjectAPI.h:72-81) ----
 * Queued in call order and applied at the start of the next step, as the reference applies its command queue in
 * Simulation::update (Simulation.cpp:39 -> ObjectManager::flushCommands / applyCommand, ObjectManager.cpp:
 * 638-790), or at once by ag2d_world_flush_commands. A command on a stale handle is dropped when applied. Every
 * command wakes the body's sleeping island. A position is the body origin's (the centre of mass moves with it); a
 * rotation is wrapped into [0, 2 pi); mass 0 makes the body static (its velocities zeroed), a positive mass scales
 * the inertia by new / old mass; an inertia is ignored on a static body. A destroyed body keeps its dense index
 * with state AG2D_BODY_DESTROYED: it is in no work list or tree, touches nothing, and its handle goes stale (the
 * reference pops it from its dense arrays instead; handles are what both keep stable). Per world: a batch
 * engine's worlds take no commands (AG2D_ERR_UNSUPPORTED). */
enum ag2d_body_state { AG2D_BODY_STATIC = 0, AG2D_BODY_SLEEPING = 1, AG2D_BODY_DYNAMIC = 2, AG2D_BODY_DESTROYED = 3 };
enum ag2d_command {
    AG2D_COMMAND_DESTROY = 0, AG2D_COMMAND_POSITION, AG2D_COMMAND_ROTATION, AG2D_COMMAND_VELOCITY,
    AG2D_COMMAND_ANGULAR_VELOCITY, AG2D_COMMAND_MASS, AG2D_COMMAND_INERTIA, AG2D_COMMAND_LOCAL_CENTER_OF_MASS,
    AG2D_COMMAND_RECOMPUTE_INERTIA, AG2D_COMMAND_MASS_FROM_DENSITY,
    /* collider commands (the handle field holds the collider's dense index) */
    AG2D_COMMAND_COLLIDER_OFFSET = 16, AG2D_COMMAND_COLLIDER_ROTATION, AG2D_COMMAND_COLLIDER_MATERIAL,
    AG2D_COMMAND_CIRCLE_RADIUS, AG2D_COMMAND_BOX_SIZE, AG2D_COMMAND_CAPSULE_SHAPE, AG2D_COMMAND_POLYGON_SHAPE
};
int32_t ag2d_world_destroy_body(ag2d_world* world, uint64_t body);
int32_t ag2d_world_set_body_position(ag2d_world* world, uint64_t body, float x, float y);
int32_t ag2d_world_set_body_rotation(ag2d_world* world, uint64_t body, float rotation);
int32_t ag2d_world_set_body_velocity(ag2d_world* world, uint64_t body, float vx, float vy);
int32_t ag2d_world_set_body_angular_velocity(ag2d_world* world, uint64_t body, float angular_velocity);
int32_t ag2d_world_set_body_mass(ag2d_world* world, uint64_t body, float mass);
int32_t ag2d_world_set_body_inertia(ag2d_world* world, uint64_t body, float inertia);
/* ObjectAPI::setBodyLocalCenterOfMass / recomputeBodyInertia / setBodyMassFromDensity (ObjectAPI.h:82-84;
 * ObjectManager.cpp:751-775, 907-970): the body origin stays put and the centre of mass moves with the local
 * centre; the inertia from the colliders' shapes at the body's mass (parallel axis to the centre of mass); the mass
 * from a density times the colliders' area. */
int32_t ag2d_world_set_body_local_center_of_mass(ag2d_world* world, uint64_t body, float x, float y);
int32_t ag2d_world_recompute_body_inertia(ag2d_world* world, uint64_t body);
int32_t ag2d_world_set_body_mass_from_density(ag2d_world* world, uint64_t body, float density);
/* ObjectAPI::setColliderLocalOffset / setColliderLocalRotation / setColliderMaterial / setCircleRadius /
 * setBoxSize / setCapsuleShape (ObjectAPI.h:86-91; ObjectManager.cpp:785-850) by dense collider index, deferred
 * like the body commands: field AG2D_COMMAND_COLLIDER_OFFSET (a, b), _ROTATION (a, wrapped into [0, 2 pi)),
 * _MATERIAL (a as the index; an unknown index becomes 0), _CIRCLE_RADIUS (a), _BOX_SIZE (a, b: width, height),
 * _CAPSULE_SHAPE (a, b: length, radius); sizes are clamped at 0, a shape setter on another shape does nothing.
 * The collider's body wakes; the body's bound radius follows. */
int32_t ag2d_world_set_collider(ag2d_world* world, uint32_t collider, int32_t command, float a, float b);
/* ObjectAPI::setPolygonShape (ObjectAPI.h:93; ObjectManager.cpp:622-636, 838-857): n collider-local vertices (xy
 * pairs) replace a polygon collider's outline. The outline is prepared at once as at creation (duplicates and
 * straight vertices dropped, made counter-clockwise); a degenerate or concave outline, or one of more than 16
 * vertices, is refused (AG2D_ERR_INVALID_ARG, the reference's false). At the next flush it is recentred on its
 * centroid, the shift added to the collider's offset (the body's mass and inertia are kept); on another shape it
 * does nothing. */
int32_t ag2d_world_set_polygon_shape(ag2d_world* world, uint32_t collider, const float* xy, uint32_t n);
/* PhysicsGeometry::preparePolygonOutline + decomposeConcave (Bayazit, ear clipping when no diagonal is valid) +
 * limitConvexPieceVertexCount (fan, 16 vertices) (PhysicsGeometry.cpp:175-212, PolygonDecomposition.cpp:704-831):
 * the convex pieces polygon creation makes from an outline, on the host (no device needed). Writes *out_pieces,
 * then the pieces' vertex counts and their vertices (xy pairs, one piece after another); AG2D_ERR_CAPACITY with
 * *out_pieces set when the arrays are too small; AG2D_ERR_INVALID_ARG for a degenerate or self-intersecting
 * outline. */
int32_t ag2d_decompose_polygon(const float* xy, uint32_t n, float* out_xy, uint32_t out_capacity,
                               uint32_t* piece_counts, uint32_t piece_capacity, uint32_t* out_pieces);

/* Applies the queued commands now (Simulation::flushCommands, Simulation.cpp:453-456). */
int32_t ag2d_world_flush_commands(ag2d_world* world);

/* ---- body constraints: ConstraintAPI (SimulationAPIs/ConstraintAPI.h:32-105) ----
 * Springs, revolute, prismatic and slider joints join two bodies at body-local anchors (a soft distance constraint
 * with a rest length; a soft pin of both anchors together; a soft lock of the translation across body A's axis and
 * of the relative angle, with optional hard limits along the axis; the same without the angle lock); a motor drives
 * one body's angular velocity toward a target speed within a torque limit. They are solved between the two halves of the step's integration, each kind in the
 * reference's dense order (Solving/SpringSolver.cpp, RevoluteJointSolver.cpp, PrismaticJointSolver.cpp,
 * SliderJointSolver.cpp, MotorSolver.cpp scheduled by
 * ConstraintScheduler.cpp:9-80): the same results as the reference's single-threaded solve. Creation wakes the
 * bodies and returns a handle (AG2D_ERR_INVALID_ARG for a stale body handle: the reference's nullopt); destruction
 * and the setters are deferred to the next step's command flush, like the body commands, and wake the bodies; a
 * destroyed body takes its constraints with it. These calls are per world (a batch's engine returns
 * AG2D_ERR_UNSUPPORTED); worlds with constraints can form a batch (each steps as alone), but not join a server or
 * a checkpoint. */
enum ag2d_joint_kind {   /* ConstraintType order */
    AG2D_JOINT_SPRING = 0, AG2D_JOINT_REVOLUTE = 1, AG2D_JOINT_PRISMATIC = 2, AG2D_JOINT_SLIDER = 3, AG2D_JOINT_MOTOR = 4
};
typedef struct ag2d_joint_desc {
    int32_t kind;                    /* ag2d_joint_kind */
    int32_t enable_limit;            /* prismatic / slider: the axis limits are enforced */
    uint64_t body_a, body_b;         /* body handles (a motor uses body_a) */
    float anchor_a_x, anchor_a_y;    /* body-local anchors (all but motors) */
    float anchor_b_x, anchor_b_y;
    float rest_length;               /* spring */
    float stiffness, damping;        /* all but motors */
    float target_speed, max_torque;  /* motor */
    float axis_x, axis_y;            /* prismatic / slider: body A's local axis (normalised; zero length: (1, 0)) */
    float lower_limit, upper_limit;  /* prismatic / slider: limits of the translation along the axis */
    float reference_angle;           /* prismatic, read only: the relative angle locked at creation */
    float impulse;                   /* motor, read only: accumulated impulse of the last step */
} ag2d_joint_desc;
/* Setter fields (ConstraintAPI::set* / reset*, ConstraintAPI.h:54-83): anchors and the axis take (a, b) as x, y (an
 * axis is normalised, a zero-length one is dropped); limits take (a, b) in either order; enable_limit takes a != 0;
 * the reference-angle reset locks the bodies' current relative angle; rest length, stiffness, damping and max
 * torque are clamped at 0 when applied. */
enum ag2d_joint_field {
    AG2D_JOINT_ANCHOR_A = 0, AG2D_JOINT_ANCHOR_B, AG2D_JOINT_REST_LENGTH, AG2D_JOINT_STIFFNESS, AG2D_JOINT_DAMPING,
    AG2D_JOINT_TARGET_SPEED, AG2D_JOINT_MAX_TORQUE, AG2D_JOINT_AXIS_A, AG2D_JOINT_LIMITS, AG2D_JOINT_ENABLE_LIMIT,
    AG2D_JOINT_RESET_REFERENCE_ANGLE
};
int32_t ag2d_world_create_joint(ag2d_world* world, const ag2d_joint_desc* desc, uint64_t* out_handle);
int32_t ag2d_world_destroy_joint(ag2d_world* world, int32_t kind, uint64_t handle);
int32_t ag2d_world_set_joint(ag2d_world* world, int32_t kind, uint64_t handle, int32_t field, float a, float b);
/* ConstraintAPI::get*DataH (ConstraintAPI.h:86-105): the constraint as stored now. AG2D_ERR_INVALID_ARG if stale. */
int32_t ag2d_world_joint(ag2d_world* world, int32_t kind, uint64_t handle, ag2d_joint_desc* out);
/* Constraints of a kind, and the handle of dense index i (ConstraintAPI::get*Handle, ConstraintAPI.h:46-50). */
int32_t ag2d_world_joint_count(ag2d_world* world, int32_t kind, uint32_t* out_count);
int32_t ag2d_world_joint_handle(ag2d_world* world, int32_t kind, uint32_t index, uint64_t* out_handle);
/* IConstraintSystem::iterations of a kind (default 6; ConstraintSystemBase.h:34). */
int32_t ag2d_world_set_joint_iterations(ag2d_world* world, int32_t kind, uint32_t iterations);

/* ---- collision events: Simulation::createCollisionCallback / destroyCollisionCallback /
 * setColliderCollisionCallback (Simulation.h:169-179, Simulation.cpp:130-171; the table of
 * SimulationImpl/CollisionCallbackManager.h) ----
 * A collider with a callback and an impulse threshold gets an event, from its side, for each manifold of a step
 * whose impact impulse (the largest over the contact points of approach speed along the normal times the normal
 * effective mass, before solving; BodyCollisionSolver.cpp:320-387) is positive and reaches the threshold. Events
 * are recorded while collision events are enabled (the default, SimulationSettings::collisionEventsEnabled,
 * Simulation.h:60) and a callback exists, and after each step the world calls each event's callback in manifold
 * order, side a before side b (the reference dispatches at the end of physicsStep, Simulation.cpp:174-180, 450;
 * here after the step's sleep pass). A callback may queue body commands and change callbacks; it may not step
 * the world. Per world: a batch engine's worlds record no events (AG2D_ERR_UNSUPPORTED). */
typedef struct ag2d_collision_event {
    uint32_t self, other;            /* dense collider indices (the reference's collider handles) */
    uint32_t self_body, other_body;  /* dense body indices */
    uint64_t self_body_handle;       /* body handles; UINT64_MAX in a world made by ag2d_world_load_state */
    uint64_t other_body_handle;
    float point_x, point_y;          /* average of the manifold's contact points */
    float normal_x, normal_y;        /* from self towards other */
    float impulse;                   /* the impact impulse */
    uint16_t callback_id;
    uint16_t pad;
} ag2d_collision_event;
typedef void (*ag2d_collision_callback)(const ag2d_collision_event* event, ag2d_world* world, void* user_data);
/* A callback slot (ids from 1; a destroyed id is reused first). AG2D_ERR_INVALID_ARG for a null function,
 * AG2D_ERR_CAPACITY when all 65,535 ids are in use (the reference returns nullopt for both). */
int32_t ag2d_world_create_collision_callback(ag2d_world* world, ag2d_collision_callback function, void* user_data,
                                             uint16_t* out_id);
/* Colliders using the id go back to no callback. AG2D_ERR_INVALID_ARG for id 0 and dead ids (reference: false). */
int32_t ag2d_world_destroy_collision_callback(ag2d_world* world, uint16_t id);
/* Id 0 clears the collider's callback (threshold ignored). AG2D_ERR_INVALID_ARG for a collider index out of range,
 * a dead id, or a threshold that is negative or NaN (reference: false). */
int32_t ag2d_world_set_collider_collision_callback(ag2d_world* world, uint32_t collider, uint16_t id,
                                                   float impulse_threshold);
/* SimulationSettings::collisionEventsEnabled (Simulation.h:59-60): 1 (the default) records events. */
int32_t ag2d_world_set_collision_events(ag2d_world* world, int32_t enable);
/* The last step's events, as dispatched (BodyCollisionSolver::getCollisionEvents, BodyCollisionSolver.h:125).
 * out_count receives the full count; at most 'capacity' events are written. */
int32_t ag2d_world_collision_events(ag2d_world* world, ag2d_collision_event* out_events, uint32_t capacity,
                                    uint32_t* out_count);

/* Replaces the world with a reference-layout state (parity harness: same inputs as the reference). */
int32_t ag2d_world_load_state(ag2d_world* world, const ag2d_state_desc* state);

/* Simulation::update with dt == the fixed interval, 'steps' times (Simulation.cpp:32-74 -> physicsStep :255-351).
 * Synchronous: returns when the steps are done and the counters are on the host. */
int32_t ag2d_world_step(ag2d_world* world, int32_t steps);

int32_t ag2d_world_counters(ag2d_world* world, ag2d_counters* out);
/* Device buffer allocations the library has made in this process so far (ag2d_counters.device_allocs). */
int32_t ag2d_device_allocs(uint64_t* out);

/* Launch-shape autotuner (no reference counterpart: the reference runs on CPU threads). Times real steps under each
 * candidate solver team size (batches), pair-query and narrow-phase block size and keeps the fastest. A step's
 * results do not depend on these settings, so tuning only advances the world: by 1 + candidates x
 * (steps_per_candidate + 1) steps, with 19 candidates for a batch and 6 for a single world. Works on a batch
 * through ag2d_batch_engine. */
int32_t ag2d_world_autotune(ag2d_world* world, int32_t steps_per_candidate, ag2d_tuning* out);
/* Applies launch shapes (for instance those the autotuner chose on a copy of the batch stepped ahead to a settled
 * state). Results do not depend on them. */
int32_t ag2d_world_set_tuning(ag2d_world* world, const ag2d_tuning* tuning);
/* Device timing of the step phases (the reference's Tracy zones, Profiling/TracyProfiler.h:66-72, become CUDA
 * events on the world's stream). Enabling resets the totals. out_ms receives cumulative milliseconds per
 * enum ag2d_timed_phase, out_calls the number of timed occurrences. */
int32_t ag2d_world_set_profiling(ag2d_world* world, int32_t enable);
int32_t ag2d_world_phase_times(ag2d_world* world, double* out_ms, uint64_t* out_calls, int32_t capacity);
/* The CUDA stream the world's kernels run on (cudaStream_t), for callers that order their own work with it. */
int32_t ag2d_world_stream(ag2d_world* world, void** out_stream);
int32_t ag2d_world_body_count(ag2d_world* world, uint32_t* out_bodies, uint32_t* out_colliders);

/* Spatial query, replacing BroadPhaseCollisionDetector::queryCollidersInShape (BroadPhaseCollisionDetector.h:
 * 189-203, BvhTree.h:110-192) with its AABBQuery and CircleQuery shapes (QueryShapes.h:8-86). Returns the indices,
 * ascending, of the colliders whose AABB as of the last step's broad phase passes the shape's test (AABB: strict
 * overlap; circle: closest-point squared distance <= radius^2, radius clamped at 0), among the trees selected by
 * 'trees' (AG2D_TREE_* bits, by the owner body's state). params: AABB {min_x, min_y, max_x, max_y}; circle
 * {x, y, radius}. Before the first step after creation or a host-side edit nothing is found (the reference's
 * trees are empty then), unless ag2d_world_load_state brought the AABBs. The reference
 * also adds every collider of a node its shape contains without the collider's own test; the sets differ only for
 * a collider AABB of zero width or height lying on the query AABB's boundary. out_count receives the full count;
 * at most 'capacity' indices are written. On a batch's engine the query covers every world of the batch. */
enum ag2d_tree_flag { AG2D_TREE_DYNAMIC = 1, AG2D_TREE_STATIC = 2, AG2D_TREE_SLEEPING = 4, AG2D_TREE_ALL = 7 };
enum ag2d_query_shape { AG2D_QUERY_AABB = 0, AG2D_QUERY_CIRCLE = 1 };
int32_t ag2d_world_query_shape(ag2d_world* world, int32_t shape, const float* params, uint32_t trees,
                               uint32_t* out_colliders, uint32_t capacity, uint32_t* out_count);
/* Colliders a circle touches, replacing NarrowPhaseCollisionDetector::findCollisionsInCircle (NarrowPhase
 * CollisionDetector.cpp:153-270) applied to what a circle query finds (ag2d_world_query_shape with
 * AG2D_QUERY_CIRCLE): a collider is reported with the signed distance from the circle's centre to its shape
 * (negative inside) when that distance is below 'radius'. Ascending indices; out_count receives the full count, at
 * most 'capacity' indices and distances are written. Same validity rule as ag2d_world_query_shape. */
int32_t ag2d_world_query_circle_contacts(ag2d_world* world, float x, float y, float radius, uint32_t trees,
                                         uint32_t* out_colliders, float* out_distance, uint32_t capacity,
                                         uint32_t* out_count);

/* Copies a field into caller memory (host). out_bytes receives the field size; pass dst = NULL to query it.
 * Replaces the reference's SoA viewers (ObjectAPI::getBodies/getColliders, ObjectAPI.h:96-101) and
 * Simulation::getBodyCollisionData (Simulation.h:186). */
int32_t ag2d_world_read(ag2d_world* world, int32_t field, void* dst, uint64_t capacity_bytes, uint64_t* out_bytes);
/* Body and collider fields (the reference's per-frame BodySoA / ColliderSoA viewers, ObjectAPI::getBodies /
 * getColliders, ObjectAPI.h:97-101, read by its renderer every frame) without waiting: the values as they stand
 * after the work queued so far are packed on the device and copied into 'dst' on a copy stream while the next
 * steps run. 'dst' must be page-locked (ag2d_host_alloc, cudaHostAlloc or cudaHostRegister) and stay untouched
 * until ag2d_world_read_wait returns. Up to four reads may be in flight; a fifth waits on the device for the first
 * one's copy. Phase-tap fields (pairs, manifolds, ...) return AG2D_ERR_UNSUPPORTED. */
int32_t ag2d_world_read_async(ag2d_world* world, int32_t field, void* dst, uint64_t capacity_bytes,
                              uint64_t* out_bytes);
/* Blocks until every ag2d_world_read_async of this world has landed in host memory. */
int32_t ag2d_world_read_wait(ag2d_world* world);
/* Page-locked host memory (cudaHostAlloc): destinations for asynchronous reads and checkpoints, one DMA per copy.
 * No reference counterpart (the reference's state lives in host memory). */
int32_t ag2d_host_alloc(uint64_t bytes, void** out_ptr);
int32_t ag2d_host_free(void* ptr);
/* Overwrites a field from host memory (body state, pairs, manifolds) for phase-level parity runs. */
int32_t ag2d_world_write(ag2d_world* world, int32_t field, const void* src, uint64_t bytes);
/* Runs one phase (enum ag2d_phase) on the current device state. */
int32_t ag2d_world_run_phase(ag2d_world* world, int32_t phase);

/* ---- batched worlds: many independent worlds advanced by one launch sequence per step ----
 * The reference runs one Simulation per world (Simulation.h:36); a batch packs the current state of several
 * worlds (same step settings) into one world-segmented device state: per-world Morton bounds, per-world trees,
 * per-world colouring and solve. Each world's result equals what it gets when stepped alone. The source worlds
 * are copied, not moved, and are not advanced by the batch. */
int32_t ag2d_batch_create(ag2d_world* const* worlds, uint32_t world_count, ag2d_batch** out_batch);
int32_t ag2d_batch_step(ag2d_batch* batch, int32_t steps);
int32_t ag2d_batch_world_count(ag2d_batch* batch, uint32_t* out_count);
/* The engine instance of the batch, for ag2d_world_counters / _stream / _set_profiling / _phase_times and
 * whole-batch reads. Owned by the batch: do not destroy it or add bodies through it. */
int32_t ag2d_batch_engine(ag2d_batch* batch, ag2d_world** out_world);
/* Reads a body field, a collider field or the manifolds of one world of the batch, in that world's own indices. */
int32_t ag2d_batch_read(ag2d_batch* batch, uint32_t world, int32_t field, void* dst, uint64_t capacity_bytes,
                        uint64_t* out_bytes);
int32_t ag2d_batch_destroy(ag2d_batch* batch);
/* Checkpoint of a batch: every resident array (body and collider state, shapes, materials, collider poses and
 * AABBs), the warm-start manifolds with their colours and the world partition, in one self-describing host blob.
 * Pass dst = NULL to get the size. A batch restored from it steps on exactly as the saved batch does (bit for bit);
 * a page-locked source (ag2d_host_alloc) goes over in one DMA per array. 'device' < 0 keeps the saved device.
 * No reference counterpart: the reference keeps its state in host memory and has no save / load of a Simulation. */
int32_t ag2d_batch_save(ag2d_batch* batch, void* dst, uint64_t capacity_bytes, uint64_t* out_bytes);
int32_t ag2d_batch_restore(const void* src, uint64_t bytes, int32_t device, ag2d_batch** out_batch);
/* Loads a checkpoint into an existing batch (same settings), reusing its device buffers where they are large
 * enough: the upload of a resident engine (a server between jobs), without allocating. */
int32_t ag2d_batch_load(ag2d_batch* batch, const void* src, uint64_t bytes);

/* ---- request server: world rollouts served from one resident, continuously repacked batch ----
 * No counterpart in the reference (it steps one Simulation per caller). A server owns one device batch and a host
 * thread. Submitted requests (a world built with the ag2d_world_add_* calls, and a step count) wait in arrival
 * order until the resident set has room under the device-memory budget (an estimate per request) and the world
 * limit; between rounds of steps, finished requests leave and waiting ones join, the batch being rebuilt on the
 * device. Each resident world advances exactly its requested number of steps, and its result is the one it gets
 * stepped alone. Latency is measured from submission to the moment the result is stored. */
typedef struct ag2d_server ag2d_server;
typedef struct ag2d_server_settings {
    ag2d_world_settings world;      /* step settings every request must share */
    uint64_t memory_budget_bytes;   /* device memory the resident requests may take (estimated per request) */
    uint32_t steps_per_round;       /* steps between admission / retirement rounds (at most; 0: 8) */
    uint32_t max_worlds;            /* resident requests at most (0: no limit) */
    uint32_t reserve_bodies;        /* size the device batch for this many resident bodies at creation (0: grow) */
    uint32_t reserved;
} ag2d_server_settings;
typedef struct ag2d_server_stats {
    uint64_t submitted, completed, waiting, resident;
    uint64_t peak_resident;          /* most requests resident at once */
    uint64_t rounds, body_steps;     /* rounds run, sum of bodies x steps of completed requests */
    double busy_ms;                  /* host time the loop spent on rounds with resident worlds */
    double step_ms, repack_ms;       /* of which: stepping, and retiring + repacking the batch */
    double p50_ms, p99_ms, max_ms;   /* completion latency of the completed requests */
} ag2d_server_stats;
enum ag2d_request_state { AG2D_REQUEST_WAITING = 0, AG2D_REQUEST_RUNNING = 1, AG2D_REQUEST_DONE = 2 };

int32_t ag2d_server_create(const ag2d_server_settings* settings, ag2d_server** out_server);
/* Copies the world's bodies into a new request; the world itself is not modified or kept. */
int32_t ag2d_server_submit(ag2d_server* server, ag2d_world* world, uint32_t steps, uint64_t* out_request);
int32_t ag2d_server_poll(ag2d_server* server, uint64_t request, int32_t* out_state, double* out_latency_ms);
/* Blocks until every submitted request is done (or the loop failed); timeout_ms < 0 waits without limit. */
int32_t ag2d_server_wait_all(ag2d_server* server, double timeout_ms);
/* A body field of a finished request (AG2D_BODY_COM_X/Y, ROTATION, VEL_X/Y, ANGULAR_VELOCITY, POSE, STATE). */
int32_t ag2d_server_read(ag2d_server* server, uint64_t request, int32_t field, void* dst, uint64_t capacity_bytes,
                         uint64_t* out_bytes);
int32_t ag2d_server_release(ag2d_server* server, uint64_t request);
int32_t ag2d_server_stats_get(ag2d_server* server, ag2d_server_stats* out_stats);
int32_t ag2d_server_destroy(ag2d_server* server);

/* ---- allocation-free solve: no counterpart in the reference (its solver allocates freely on the host) ----
 * Colours and solves n_manifolds manifolds in place on caller-owned device arrays: body velocities and poses are
 * updated and the manifolds' impulses written back, as AG2D_PHASE_SOLVE does for a world. The call makes no device
 * allocation and no allocating library call. It is for callers that cannot allocate at this point: a host loop
 * that has handed all free device memory to its own pool and runs inside that budget, or code that must not stall
 * a busy device on the implicit synchronisation that cudaMalloc / cudaFree can bring. Its scratch is one fixed
 * static device array of about 3.1 MiB per device, so:
 *  - at most AG2D_SOLVE_NOALLOC_MAX_MANIFOLDS manifolds and AG2D_SOLVE_NOALLOC_MAX_BODIES bodies per call; larger
 *    sizes return AG2D_ERR_CAPACITY with the limit in the error string, before any launch;
 *  - the array's address belongs to a CUDA context: the first call in each context (the first on a device, and the
 *    first again after cudaDeviceReset or when another context is made current on that device) looks it up
 *    (cudaGetSymbolAddress) and caches it under the context's unique id, so that call performs set-up; make it
 *    before any stream capture in that context;
 *  - a CUDA error already pending when the call starts (left by the caller's earlier work) is returned as
 *    AG2D_ERR_CUDA without launching and is left pending, so a launch error reported here is this call's own;
 *  - the kernel clears what it needs at the start of every call: nothing has to start at zero;
 *  - calls that overlap on one device share the array and race: serialise them (one stream, or events).
 * The call is asynchronous on 'stream' (a cudaStream_t, NULL for the default stream) on the current device.
 * Layout: body_velocity [n_bodies][4] = vx, vy, angular velocity, inverse mass; body_pose [n_bodies][4] =
 * x, y, rotation, inverse inertia; materials [n_materials][4] = elasticity, static friction, dynamic friction,
 * unused; collider_body / collider_material index those arrays and must be in range. Float4 arrays and the
 * manifolds must be 16-byte aligned. device_status (device memory, may be NULL) receives {status bits, colours}. */
#define AG2D_SOLVE_NOALLOC_MAX_MANIFOLDS 16384u
#define AG2D_SOLVE_NOALLOC_MAX_BODIES 16384u
typedef struct ag2d_solve_view {
    uint32_t n_bodies;
    float* body_velocity;
    float* body_pose;
    uint32_t n_colliders;
    const uint32_t* collider_body;
    const uint32_t* collider_material;
    uint32_t n_materials;
    const float* materials;
} ag2d_solve_view;
int32_t ag2d_solve_noalloc(const ag2d_solve_view* view, ag2d_manifold* manifolds, uint32_t n_manifolds,
                           uint32_t velocity_iterations, uint32_t position_iterations, void* stream,
                           uint32_t* device_status);

#ifdef __cplusplus
}
#endif
#endif
