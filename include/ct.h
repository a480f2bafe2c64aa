/* ct.h -- C ABI of the B200 voxel ray-tracing hot path (cube-tracing
 * compatible).
 *
 * The entry points replace the two Vulkan ray-tracing dispatches, the TAA
 * compute dispatch and the acceleration-structure build of cube-tracing:
 *
 *   ct_build_accel   <- ACCEL_STRUCT_MNGR::build_blases / build_tlas
 *                       (src/accel_struct_mngr.cpp:1362-1504, 1854-1973)
 *   ct_trace_frame   <- pass 1 of rgen.glsl up to the DI info
 *                       (src/shaders/glsl/raytracing/rgen.glsl:46-201, 319;
 *                        recorded at src/main.cpp:1570-1589)
 *   ct_restir_di     <- stage 0: rest of pass 1, RIS + visibility + temporal
 *                       reuse (rgen.glsl:203-268);
 *                       stage 1: pass 2, spatial reuse + shading
 *                       (rgen.glsl:329-510; src/main.cpp:1596-1615)
 *   ct_taa           <- src/shaders/glsl/compute/taa.glsl:16-109
 *                       (src/main.cpp:1617-1651)
 *   ct_render_frame  <- the sequence App::draw records (src/main.cpp:1436-1703)
 *
 * Every call is stream ordered and asynchronous: arguments are checked on
 * the host, kernels are enqueued on `stream`, and the call returns.  All
 * buffers are owned by the caller and passed as device addresses, laid out
 * exactly as the reference's GPU structs (src/shaders/shared.inl, Daxa
 * scalar block layout); ct_accel is the only object the library allocates.
 * No function throws, aborts or prints; errors come back as ct_status codes,
 * and errors detected on the device are latched into a device status word
 * read by ct_get_error.
 */
#ifndef CT_H
#define CT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CT_ABI_VERSION 1u

typedef struct CUstream_st *ct_stream; /* a cudaStream_t; NULL = legacy default stream */

typedef enum ct_status {
  CT_OK = 0,
  CT_ERR_INVALID_ARG = 1,   /* null pointer, zero size, bad enum, misaligned buffer */
  CT_ERR_CAPACITY = 2,      /* a count above the supported maximum */
  CT_ERR_CUDA = 3,          /* a CUDA runtime call failed (see ct_last_cuda_error) */
  CT_ERR_ITER_LIMIT = 4,    /* a device loop hit its iteration cap (device latched) */
  CT_ERR_NAN_INPUT = 5,     /* non-finite camera or scene data */
  CT_ERR_UNSUPPORTED = 6,   /* a feature the hot path does not implement */
  CT_ERR_NOT_GRID_ALIGNED = 7 /* an AABB is not one voxel of the instance grid */
} ct_status;

/* ---------------------------------------------------------------------------
 * Reference GPU structs (src/shaders/shared.inl).  Field names and order are
 * the reference's; vectors are written as float[3] (scalar layout: 4-byte
 * aligned, no padding), 64-bit addresses are 8-byte aligned.
 */
typedef struct ct_aabb { float minimum[3]; float maximum[3]; } ct_aabb;                       /* AABB, 24 B   */
typedef struct ct_object_info { uint32_t instance_id; uint32_t primitive_id; } ct_object_info; /* OBJECT_INFO  */
typedef struct ct_instance {                                                                    /* INSTANCE, 72 B */
  float transform[16];            /* column major object-to-world */
  uint32_t first_primitive_index;
  uint32_t primitive_count;
} ct_instance;
typedef struct ct_primitive { uint32_t material_index; uint32_t light_index; } ct_primitive;    /* PRIMITIVE, 8 B */
typedef struct ct_material {                                                                    /* MATERIAL, 84 B */
  uint32_t type;                  /* low 8 bits: 0 lambertian, 1 metal, 2 dielectric, 3 constant medium */
  float ambient[3], diffuse[3], specular[3], transmittance[3], emission[3];
  float shininess, roughness, ior, dissolve;
  int32_t illum;
} ct_material;
typedef struct ct_light {                                                                       /* LIGHT, 40 B */
  float position[3];
  float emissive[3];
  ct_object_info instance_info;
  float size;
  uint32_t type;                  /* CT_LIGHT_* */
} ct_light;
typedef struct ct_light_config {                                                                /* LIGHT_CONFIG, 52 B */
  uint32_t point_light_count; float point_light_pdf;
  uint32_t cube_light_count; float cube_light_pdf;
  uint32_t sphere_light_count; float sphere_light_pdf;
  uint32_t analytic_light_count; float analytic_light_pdf;
  uint32_t env_map_count; float env_map_pdf;
  uint32_t brdf_count; float brdf_pdf;
  uint32_t light_count;
} ct_light_config;
typedef struct ct_reservoir {                                                                   /* RESERVOIR, 36 B */
  uint32_t Y, l_type, seed;
  float W_y, W_sum, M;
  float F[3];
} ct_reservoir;
typedef struct ct_object_hit { ct_object_info object; float hit[3]; } ct_object_hit;            /* OBJECT_HIT, 20 B */
typedef struct ct_path_reservoir {                                                              /* PATH_RESERVOIR, 92 B */
  float M, weight;
  uint32_t path_flags, rc_random_seed;
  float F[3];
  float light_pdf;
  float cached_jacobian[3];
  uint32_t init_random_seed;
  ct_object_hit rc_vertex_hit;
  float rc_vertex_wi[3];
  float rc_vertex_irradiance[3];
} ct_path_reservoir;
typedef struct ct_velocity { float velocity[2]; } ct_velocity;                                  /* VELOCITY, 8 B */
typedef struct ct_di_info {                                                                     /* DIRECT_ILLUMINATION_INFO, 60 B */
  float position[3];
  float distance;
  float normal[3];
  float ray_origin[3];
  uint32_t seed;
  ct_object_info instance_hit;
  uint32_t mat_index;
  float confidence;
} ct_di_info;
typedef struct ct_camera_view {                                                                 /* camera_view, 264 B */
  float inv_view[16], inv_proj[16];
  float defocus_angle, focus_dist;
  float prev_inv_view[16], prev_inv_proj[16];
} ct_camera_view;
typedef struct ct_status_block {                                                                /* Status, 96 B */
  uint32_t resolution[2];
  uint32_t frame_number;
  uint32_t _pad0;
  uint64_t num_accumulated_frames;
  uint32_t pixel[2];
  uint32_t is_active;             /* CT_*_BIT feature bits */
  uint32_t _pad1;
  uint64_t light_config_address;  /* device address of ct_light_config */
  uint32_t obj_count;
  float time;
  uint32_t is_afternoon;
  uint32_t max_depth;
  uint64_t brush_config_address, brush_counter_address, instance_bitmask_address, primitive_bitmask_address;
} ct_status_block;
typedef struct ct_world {                                                                       /* WORLD, 96 B: device addresses */
  uint64_t instance_address, instance_address_prev;
  uint64_t primitive_address, primitive_address_prev;
  uint64_t aabb_address, aabb_address_prev;
  uint64_t remapped_primitive_address, remapped_cube_light_address;
  uint64_t material_address;
  uint64_t point_light_address, cube_light_address, env_light_address;
} ct_world;
typedef struct ct_restir {                                                                      /* RESTIR, 72 B: device addresses */
  uint64_t previous_reservoir_address;
  uint64_t intermediate_reservoir_address;
  uint64_t reservoir_address;
  uint64_t previous_di_address;
  uint64_t di_address;
  uint64_t velocity_address;
  uint64_t output_path_reservoir_address;
  uint64_t temporal_path_reservoir_address;
  uint64_t indirect_color_address;
} ct_restir;

/* Voxel brush records (shared.inl:220-231). */
typedef struct ct_brush_config {                                                                /* BRUSH_CONFIG, 28 B */
  uint32_t brush_type;             /* CT_BRUSH_TYPE_SQUARE */
  float brush_size[3];
  uint32_t brush_pixel_size[3];    /* [0]: half width of the screen window, pixels */
} ct_brush_config;
typedef struct ct_brush_counter { uint32_t instance_count, primitive_count; } ct_brush_counter;  /* BRUSH_COUNTER, 8 B */
#define CT_BRUSH_TYPE_SQUARE 0u

/* Feature bits of ct_status_block.is_active (shared.inl:73-79). */
#define CT_TAA_BIT (1u << 0)
#define CT_RIS_POINT_LIGHT_BIT (1u << 1)
#define CT_RIS_ENV_LIGHT_BIT (1u << 2)
#define CT_RIS_CUBE_LIGHT_BIT (1u << 3)
#define CT_RIS_BRDF_BIT (1u << 4)
#define CT_REMAP_BIT (1u << 30)

/* LIGHT.type values (shared.inl:336-342). */
#define CT_LIGHT_NONE 0u
#define CT_LIGHT_POINT 1u
#define CT_LIGHT_CUBE 2u
#define CT_LIGHT_ENV_MAP 5u

/* Invalid-id sentinels (shared.inl:18-20). */
#define CT_MAX_INSTANCES 983040u
#define CT_MAX_PRIMITIVES 134217728u
#define CT_MAX_MATERIALS 10000u

/* ---------------------------------------------------------------------------
 * Push constant of every pass (PushConstant, shared.inl:442-455).  Images
 * are headless RGBA32F buffers of size[0]*size[1] texels, row major.
 */
typedef struct ct_accel ct_accel;
typedef struct ct_push_constant {
  uint32_t size[2];
  const ct_accel *tlas;            /* current scene */
  const ct_accel *tlas_previous;   /* previous frame's scene (may equal tlas) */
  float *swapchain;                /* output image of this frame */
  const float *previous_swapchain; /* output image of the previous frame (TAA history) */
  float *taa_frame;                /* shaded image before TAA */
  float *taa_prev_frame;           /* unused by the hot path, kept for layout */
  uint64_t camera_buffer;          /* device address of ct_camera_view */
  uint64_t status_buffer;          /* device address of ct_status_block */
  uint64_t world_buffer;           /* device address of ct_world */
  uint64_t restir_buffer;          /* device address of ct_restir */
} ct_push_constant;

/* ---------------------------------------------------------------------------
 * Run-time parameters.  The reference fixes these at shader compile time
 * (src/shaders/include/defines.glsl:34-62, shared.inl:45, taa.glsl:13);
 * ct_params_default() returns exactly those values.
 */
#define CT_MAX_NEIGHBORS 8u
typedef struct ct_params {
  uint32_t struct_size;            /* sizeof(ct_params) */
  float voxel_extent;              /* VOXEL_EXTENT: edge of one voxel, object units */
  uint32_t min_ris_point_samples, max_ris_point_samples;
  uint32_t min_ris_env_samples, max_ris_env_samples;
  uint32_t min_ris_cube_samples, max_ris_cube_samples;
  float min_influence_from_the_past, max_influence_from_the_past;
  uint32_t min_num_of_neighbors, max_num_of_neighbors; /* <= CT_MAX_NEIGHBORS */
  float min_neighbors_radius, max_neighbors_radius;
  float max_distance_to_hit;
  uint32_t spatial_passes;         /* 1 in the reference; >1 adds passes before shading */
  float taa_alpha;                 /* weight of the current frame, ALPHA in taa.glsl */
  uint32_t flags;                  /* CT_PARAM_* */
  uint32_t pt_neighbor_count;      /* ReSTIR PT spatial reuse: NEIGHBOR_COUNT (defines.glsl:61) */
  int32_t pt_neighbor_radius;      /* NEIGHBOR_RADIUS, pixels (defines.glsl:62) */
  float pt_max_influence_from_the_past; /* MAX_INFLUENCE_FROM_THE_PAST_THRESHOLD_PT (defines.glsl:58) */
  uint32_t walk_step_limit;        /* 0: the built-in cap (65536 cells per walk); a smaller cap makes long walks
                                      end with CT_ERR_ITER_LIMIT, to exercise that path (ct_trace_frame,
                                      ct_restir_di, ct_restir_pt) */
  uint64_t counters_address;       /* optional device uint64[CT_COUNTER_COUNT] counters (CT_COUNTER_*) */
  uint64_t workspace_address;      /* optional caller scratch for ct_restir_di (ct_workspace_size bytes, */
  uint64_t workspace_bytes;        /* 256-byte aligned); 0 = scratch owned by the acceleration structure */
  uint32_t walker_blocks;          /* blocks of 256 threads of the persistent ray walkers (shadow rays, PT
                                      bounce rays); 0: 8 per SM.  A schedule knob for views rendered side by
                                      side (ct_render_views); results do not depend on it */
  uint32_t pt_shift_mapping;       /* ReSTIR PT shift: CT_SHIFT_RECONNECTION (the reference's, rgen.glsl:282,
                                      437) or CT_SHIFT_HYBRID (reconnection after a random-number replay of
                                      the prefix, with the reconnection vertex chosen as the first vertex
                                      whose incoming segment is at least pt_near_field_distance long and
                                      which, with its predecessor, is rough; path_tracer.glsl:478-516) */
  float pt_near_field_distance;    /* NEAR_FIELD_DISTANCE (defines.glsl:53); 0: HALF_VOXEL_EXTENT * 0.5 */
  uint32_t _reserved;              /* 0 */
} ct_params;
#define CT_SHIFT_RECONNECTION 0u   /* SHIFT_MAPPING_RECONNECTION (defines.glsl:86) */
#define CT_SHIFT_HYBRID 2u         /* SHIFT_MAPPING_HYBRID (defines.glsl:88) */

#define CT_PARAM_COUNT_RAYS (1u << 0) /* accumulate work counters into counters_address */
/* The frame includes indirect illumination (ReSTIR PT): the switch the
 * reference sets at compile time as INDIRECT_ILLUMINATION_ON
 * (defines.glsl:20).  With it, ct_trace_frame clears the indirect colour of
 * missed pixels (rgen.glsl:174-176), ct_restir_di(stage 1) leaves the final
 * shading to ct_restir_pt(stage 1), and ct_render_frame runs the PT stages. */
#define CT_PARAM_INDIRECT (1u << 1)

/* counters_address: uint64[CT_COUNTER_COUNT], added to by every launch */
#define CT_COUNTER_PRIMARY 0      /* camera rays */
#define CT_COUNTER_SHADOW 1       /* visibility (shadow) rays */
#define CT_COUNTER_BOUNCE 2       /* closest-hit queries from surfaces */
#define CT_COUNTER_VOXEL_TESTS 3  /* ray / voxel box tests */
#define CT_COUNTER_BRICK_VISITS 4 /* 8^3 bricks entered by the walks */
#define CT_COUNTER_CANDIDATES 5   /* RIS light candidates evaluated */
#define CT_COUNTER_NEIGHBOURS 6   /* neighbour (DI, reservoir) records read by spatial reuse */
#define CT_COUNTER_TEMPORAL 7     /* previous-frame (DI, material) records read by temporal reuse */
#define CT_COUNTER_HITS 8         /* pixels with a primary hit that the launch shaded */
#define CT_COUNTER_BOUNCE_HITS 9  /* closest-hit queries from surfaces that hit a voxel */
#define CT_COUNTER_WALKER_BRICKS 10 /* of CT_COUNTER_BRICK_VISITS: bricks the shadow-ray walker entered */
#define CT_COUNTER_COUNT 11

/* ---------------------------------------------------------------------------
 * Scene description for ct_build_accel: device addresses of the caller's
 * INSTANCE / AABB buffers (the same buffers WORLD points at).  Every AABB of
 * an instance must be one voxel of a grid of edge voxel_extent in that
 * instance's object space (minimum = integer * voxel_extent,
 * maximum = minimum + voxel_extent), which is what the reference's loader
 * produces (src/gvox/map_loader.cpp:264-272).
 */
typedef struct ct_scene_desc {
  uint64_t instance_address;       /* ct_instance[instance_count] */
  uint32_t instance_count;
  uint32_t _pad;
  uint64_t aabb_address;           /* ct_aabb[aabb_count] */
  uint32_t aabb_count;
  float voxel_extent;
} ct_scene_desc;

typedef struct ct_accel_info {
  uint32_t instance_count;
  uint32_t brick_count;            /* occupied 8^3 bricks over all instances */
  uint32_t voxel_count;            /* distinct occupied voxels */
  uint32_t grid_exact;             /* 1 when voxel centres are recomputed exactly from integer coordinates */
  uint64_t device_bytes;           /* bytes the accel holds on the device */
  int32_t grid_min[3], grid_dim[3];/* voxel bounds of instance 0 */
} ct_accel_info;

typedef struct ct_error_info {
  ct_status status;                /* first device error since the last reset */
  uint32_t detail;                 /* which loop or check */
  uint32_t pixel;                  /* linear pixel index, when known */
  uint32_t _pad;
} ct_error_info;

/* ---------------------------------------------------------------------------
 * Entry points
 */
uint32_t ct_abi_version(void);
const char *ct_status_string(ct_status s);
/* Last CUDA error string seen by this thread (after CT_ERR_CUDA). */
const char *ct_last_cuda_error(void);
void ct_params_default(ct_params *out);

/* Builds the voxel acceleration structure (one brick map per instance, bricks
 * of 8^3 voxels with a 512-bit occupancy mask and a voxel -> primitive table)
 * from the caller's INSTANCE and AABB buffers.  Synchronises `stream` once to
 * size the allocation.  Duplicate voxels keep the lowest primitive id. */
ct_status ct_build_accel(const ct_scene_desc *scene, ct_accel **out_accel, ct_stream stream);
ct_status ct_accel_get_info(const ct_accel *accel, ct_accel_info *out);
ct_status ct_accel_free(ct_accel *accel);
/* The walk's cell field of one instance's grid for one ray octant (bit 0: x
 * decreasing, bit 1: y, bit 2: z), decoded: one byte per cell, x fastest,
 * the edge of the cube without occupied cells that the walk may take from
 * that cell (0 = occupied).  Writes the grid's first voxel coordinate to
 * grid_min and its cells per axis to cells; `edges` (device memory of
 * cells[0] * cells[1] * cells[2] bytes, written on `stream`) may be NULL to
 * ask for those alone.  For tests and tools; no reference counterpart. */
ct_status ct_accel_field(const ct_accel *accel, uint32_t instance, uint32_t octant, uint8_t *edges,
                         int32_t grid_min[3], uint32_t cells[3], ct_stream stream);

/* Bytes of scratch ct_restir_di needs for a width x height frame with these
 * parameters: the shadow-ray queue of one wavefront round and one answer byte
 * per (pixel, shadow-ray call site).  Pass a buffer of that size in
 * ct_params.workspace_address, or leave it 0 and the library keeps one per
 * acceleration structure (calls that share a ct_accel must then be ordered
 * on one stream). */
ct_status ct_workspace_size(uint32_t width, uint32_t height, const ct_params *params, uint64_t *out_bytes);

/* Pass 1, front half: primary rays, closest hit, motion vectors, DI info;
 * sky colour into swapchain (and taa_frame when TAA_BIT) for missed pixels. */
ct_status ct_trace_frame(const ct_push_constant *pc, const ct_params *params, ct_stream stream);
/* stage 0: RIS over the active light types + visibility + temporal reuse.
 * stage 1: spatial reuse (params->spatial_passes rounds) + shading. */
ct_status ct_restir_di(const ct_push_constant *pc, const ct_params *params, int stage, ct_stream stream);
/* ReSTIR PT (src/shaders/glsl/restir_pt/*.glsl) with the reconnection shift
 * the reference's ray-generation shader selects (SHIFT_MAPPING_RECONNECTION,
 * rgen.glsl:282, 437).  Requires CT_PARAM_INDIRECT in params->flags.
 *   stage 0: per hit pixel, a path from the primary hit with next-event
 *            estimation towards the point lights, the path reservoir, and
 *            temporal path reuse (indirect_illumination_restir_path_tracing,
 *            indirect_illumination.glsl:283-305); writes
 *            RESTIR.output_path_reservoir, RESTIR.indirect_color and the DI
 *            seed.  Call after ct_restir_di(stage 0): pass 1, rgen.glsl:271-315.
 *   stage 1: spatial path reuse (indirect_illumination_spatial_reuse,
 *            indirect_illumination.glsl:309-452) and the pixel's final
 *            shading; writes RESTIR.temporal_path_reservoir and the images.
 *            Call after ct_restir_di(stage 1): pass 2, rgen.glsl:427-452. */
ct_status ct_restir_pt(const ct_push_constant *pc, const ct_params *params, int stage, ct_stream stream);

/* Per-kernel timing for profiling (no reference counterpart; diagnostics).
 * While enabled, every kernel the library launches is bracketed by two CUDA
 * events recorded on its stream.  ct_profile_read waits for the recorded
 * events and returns one entry per kernel that ran (name, summed event
 * time in ms, launch count); `count` receives the number of entries, of
 * which at most `capacity` are written.  The timing adds two event records
 * per launch: leave it off for headline measurements. */
typedef struct ct_kernel_time {
  const char *name;
  double total_ms;
  uint64_t launches;
} ct_kernel_time;
ct_status ct_profile_enable(int enable);
ct_status ct_profile_read(ct_kernel_time *out, uint32_t capacity, uint32_t *count, int reset);

/* ct_restir_di with its scratch taken from a fixed array inside the library
 * instead of ct_params.workspace_address or a cudaMalloc'd buffer.  This
 * entry point has no counterpart in the reference: it exists for hosts that
 * cannot allocate device memory at frame time (fixed arenas set up at start,
 * no device-wide synchronisation allowed, plug-in hosts that own every
 * allocation).  It allocates nothing.  Frames whose scratch
 * (ct_workspace_size) exceeds CT_STATIC_WORKSPACE_BYTES -- e.g. above
 * 256x256 pixels with the default four spatial neighbours -- return
 * CT_ERR_CAPACITY.  Every GPU that loads the library holds the array until
 * the process exits; all calls share it, so calls that overlap on the GPU
 * race -- order them on one stream.  The first call on a device looks the
 * array up for that device; make it before any stream capture. */
#define CT_STATIC_WORKSPACE_BYTES (40u << 20)
ct_status ct_restir_di_static(const ct_push_constant *pc, const ct_params *params, int stage, ct_stream stream);

/* Frame history checkpoint (no reference counterpart: the reference keeps
 * its history only in its GPU buffers, main.cpp:96-120).  The state one frame
 * leaves for the next is every per-pixel buffer the RESTIR table names and
 * the push constant's four images.  ct_state_save writes them behind a
 * 128-byte header, each in the layout the buffers have (the reference's
 * AoS structs and RGBA32F images), in this order:
 *   previous_reservoir, intermediate_reservoir, reservoir, previous_di, di,
 *   velocity, output_path_reservoir, temporal_path_reservoir,
 *   indirect_color; swapchain, previous_swapchain, taa_frame,
 *   taa_prev_frame.
 * ct_state_load writes a blob saved for the same size back into the buffers
 * that pc names, section by section, image by role.  A renderer that loads
 * the state saved after frame k and renders frame k+1 with the same camera,
 * Status and scene continues the saved run exactly.  `blob` may be host
 * memory (pageable or pinned) or device memory.  Both calls return when
 * their copies are complete.  CT_ERR_INVALID_ARG: a null pointer, a size
 * other than ct_state_size's, or (load) a header that is not a saved state
 * of this frame size.  ct_state_size needs no device. */
#define CT_STATE_MAGIC 0x54535443u  /* "CTST" */
#define CT_STATE_VERSION 1u
#define CT_STATE_HEADER_BYTES 128u
#define CT_STATE_SECTIONS 13u
ct_status ct_state_size(uint32_t width, uint32_t height, uint64_t *out_bytes);
ct_status ct_state_save(const ct_push_constant *pc, void *blob, uint64_t bytes, ct_stream stream);
ct_status ct_state_load(const ct_push_constant *pc, const void *blob, uint64_t bytes, ct_stream stream);

/* Spatial 3x3 filter + reprojected history (taa.glsl); dispatches
 * (W/8)x(H/8) groups like the reference, so edge pixels past the last full
 * 8x8 tile are left untouched. */
ct_status ct_taa(const ct_push_constant *pc, const ct_params *params, ct_stream stream);
/* The whole frame in the reference's order: trace, DI stage 0, DI stage 1,
 * and TAA when the status block's is_active has CT_TAA_BIT.  `is_active` is
 * the host copy of that word (the library does not read device memory back). */
ct_status ct_render_frame(const ct_push_constant *pc, const ct_params *params, uint32_t is_active, ct_stream stream);

/* Many views rendered side by side (no counterpart in the reference, which
 * renders one view per frame).  Each view is a whole frame of its own --
 * push constant, parameters, status word -- recorded as ct_render_frame
 * records it, on the stream lanes[view.lane]: the lanes first wait for the
 * work already on `stream`, and `stream` then waits for every lane, so the
 * call is one stream-ordered step of `stream` and can be captured into a
 * CUDA graph (one graph launch then renders every view, the lanes becoming
 * independent branches the GPU runs concurrently).  n_lanes == 0 records
 * every view on `stream` in order.  With lanes, every view needs its own
 * scratch (params.workspace_address) and per-pixel buffers; views may share
 * an acceleration structure and scene buffers.  The first call on a device
 * creates the library's fork/join events for it; make it before capturing.
 * Results are those of n_views separate ct_render_frame calls. */
typedef struct ct_view {
  ct_push_constant pc;
  ct_params params;
  uint32_t is_active;              /* host copy of the view's Status.is_active */
  uint32_t lane;                   /* index into lanes (ignored when n_lanes == 0) */
} ct_view;
#define CT_MAX_LANES 64u
ct_status ct_render_views(const ct_view *views, uint32_t n_views, const ct_stream *lanes, uint32_t n_lanes,
                          ct_stream stream);

/* Batch ray queries against an acceleration structure, with the hit rules
 * the frame passes use.  `queries` and `results` are device arrays of n
 * entries.
 *   ct_trace_visibility: is_vertex_visible (light.glsl:82-142): result 1 when
 *     no voxel other than the target blocks [0, distance] of the ray;
 *     CT_QUERY_CHECK_TARGET in flags makes the target voxel
 *     (target_instance, target_primitive) transparent.
 *   ct_trace_closest: closest hit of the intersection shader (rint.glsl):
 *     result = (instance, primitive, t) or instance = CT_MAX_INSTANCES on a
 *     miss; ties go to the lowest primitive index. */
typedef struct ct_ray_query {
  float origin[3];
  float distance;          /* visibility: segment length; closest: t_max */
  float direction[3];
  uint32_t flags;          /* CT_QUERY_* */
  uint32_t target_instance;
  uint32_t target_primitive;
} ct_ray_query;            /* 40 B */
#define CT_QUERY_CHECK_TARGET 1u
typedef struct ct_ray_hit { uint32_t instance_id, primitive_id; float t; uint32_t _pad; } ct_ray_hit;
ct_status ct_trace_visibility(const ct_accel *accel, const ct_ray_query *queries, uint32_t n, uint8_t *results,
                              ct_stream stream);
ct_status ct_trace_closest(const ct_accel *accel, const ct_ray_query *queries, uint32_t n, ct_ray_hit *results,
                           ct_stream stream);

/* ---------------------------------------------------------------------------
 * Scene edits: the voxel brush and the primitive rearrangement that
 * cube-tracing records in its brush task graph
 * (ACCEL_STRUCT_MNGR::check_voxel_modifications, accel_struct_mngr.cpp:2802-2830),
 * followed by a rebuild of the acceleration structure.  A frame rendered
 * after an edit with CT_REMAP_BIT in the status block, the rebuilt structure
 * in pc->tlas and the one before the edit in pc->tlas_previous, reuses the
 * previous frame's reservoirs through the remap tables (TEMPORAL_REUSE,
 * restir_resampling.glsl:311-416).
 *
 * ct_brush <- entry_brush (src/shaders/slang/compute/squared_brush.slang:74-133).
 *   One thread per pixel of Status.resolution.  When the previous frame's DI
 *   record at Status.pixel is a hit, every pixel of the square window
 *   [pixel - w, pixel + w] (w = BRUSH_CONFIG.brush_pixel_size[0]; the lower
 *   corner computed in unsigned 32-bit arithmetic as the shader does, so a
 *   window that would cross the left or top edge selects nothing) whose
 *   previous DI record hits the same instance marks its primitive: bit
 *   (first_primitive_index + primitive_id) of Status.primitive_bitmask_address,
 *   bit instance_id of Status.instance_bitmask_address, and one count per
 *   newly set bit in the BRUSH_COUNTER at Status.brush_counter_address.
 *
 * ct_rearrange <- entry_rearragement (rearrangement.slang:56-204) with the
 *   host bookkeeping around it (process_voxel_modifications,
 *   restore_bitmask_buffers, accel_struct_mngr.cpp:2679-2800, and the cube
 *   light removal of delete_aabb_device_buffer / update_light_remapping_buffer,
 *   :607-816).  For every instance with marked primitives (k of its n), the
 *   marked primitives are removed and the instance stays dense: the j-th
 *   marked primitive below n - k receives the PRIMITIVE and AABB of the j-th
 *   unmarked primitive at or above n - k, INSTANCE.primitive_count becomes
 *   n - k, and WORLD.remapped_primitive_address (int32 per global primitive)
 *   gets -1 at every marked primitive and the new instance-relative index at
 *   every moved one.  Cube lights of marked primitives are removed the same
 *   way over the LIGHT_CONFIG.cube_light_count lights (moved lights keep
 *   their PRIMITIVE.light_index and LIGHT.instance_info in step;
 *   WORLD.remapped_cube_light_address gets -1 / the new index; cube_light_count
 *   and light_count drop by the removed lights).  For a single marked
 *   primitive this is the reference's swap with the last primitive.  Both
 *   remap tables must be zero on entry (their state after the frame that
 *   consumed the previous edit, when the host clears them as the reference's
 *   settling step does).  Finally both bitmasks (instance_count and
 *   primitive_count bits) and the counter are cleared.  Rebuild the
 *   acceleration structure from the same INSTANCE/AABB buffers afterwards.
 */
ct_status ct_brush(const ct_push_constant *pc, ct_stream stream);
ct_status ct_rearrange(const ct_push_constant *pc, uint32_t instance_count, uint32_t primitive_count,
                       ct_stream stream);

/* ---------------------------------------------------------------------------
 * Path-replay adjoint of a plain path tracer over per-voxel albedo and
 * emission (no counterpart in the reference, whose renderer is not
 * differentiable).  The forward model is the reference's Lambertian
 * scatter: camera rays and bounce rays take the closest voxel with the rules
 * of intersect() (bounce.glsl:9-125), each hit voxel v adds emission E[v]
 * times the path throughput, and a bounce continues in a cosine-weighted
 * direction (random_cosine_direction, prng.glsl:84-106; rcall_scatter.glsl:74-86)
 * from the hit point moved off the surface twice (compute_ray_origin,
 * primitives.glsl:233-257), which makes the throughput factor of
 * evaluate_material / sample_material_pdf (mat.glsl:66-88, light.glsl:200-229)
 * the voxel's albedo a[v].  A path has at most max_depth surface vertices
 * (the primary hit is the first); a ray that misses ends the path and adds
 * miss_radiance (0 for the adjoint's workload) times the throughput.  Per
 * pixel, without miss light:
 *   image = (1/spp) sum_s sum_k (prod_{i<k} a[v_i]) E[v_k]
 * Sample s of pixel p draws from the LCG (random.glsl:43-77) seeded with
 * tea(p, seed + s): two numbers jitter the camera ray inside the pixel, two
 * per bounce choose the direction.  Those counters are all a path needs to
 * be traced again, so ct_adjoint_backward replays each path from them and
 * stores no vertices: it accumulates
 *   d_albedo[v]   += sum over vertices v_k = v of  g . T_k . S_k
 *   d_emission[e] += sum over vertices v_k = v of  g . T_k      (e = emitter slot of v)
 * where g = d_image[p] / spp, T_k = prod_{i<k} a[v_i] and S_k is the
 * radiance the path gathers after v_k (S_k = a[v_{k+1}] S_{k+1} + E[v_{k+1}]).
 * Gradients are added with atomics, so their last bits depend on the order.
 * albedo: float[primitive_count * 3] by global primitive index
 * (INSTANCE.first_primitive_index + primitive id); emitter_index:
 * int32[primitive_count], the voxel's row of `emission` (float[emitter_count
 * * 3]) or -1.  image / d_image: float[height * width * 3] (or double with
 * CT_ADJOINT_IMAGE_F64, for finite differences), row-major; only the pixels
 * of `rect` are traced (and, forward, written).  The camera is a
 * ct_camera_view (inv_view, inv_proj) in device memory.  All pointers are
 * device memory.  CT_ERR_INVALID_ARG: a null pointer, zero sizes, spp or
 * max_depth out of range, a rect outside the frame. */
#define CT_ADJOINT_MAX_DEPTH 16u
#define CT_ADJOINT_IMAGE_F64 (1u << 0)
typedef struct ct_adjoint_desc {
  uint32_t struct_size;            /* sizeof(ct_adjoint_desc) */
  uint32_t width, height;
  uint32_t spp;                    /* samples per pixel, 1..65536 */
  uint32_t max_depth;              /* surface vertices per path, 1..CT_ADJOINT_MAX_DEPTH */
  uint32_t seed;                   /* frame seed of the sample streams */
  uint32_t flags;                  /* CT_ADJOINT_* */
  uint32_t primitive_count;        /* rows of albedo / emitter_index */
  uint32_t emitter_count;          /* rows of emission */
  uint32_t rect[4];                /* x0, y0, x1, y1 (exclusive); x1 == 0: the whole frame */
  float miss_radiance;             /* grey radiance of rays that leave the scene (0: none) */
  uint64_t camera_address;         /* ct_camera_view */
  uint64_t emitter_index_address;  /* int32[primitive_count] */
} ct_adjoint_desc;
ct_status ct_adjoint_forward(const ct_accel *accel, const ct_adjoint_desc *desc, const float *albedo,
                             const float *emission, void *image, ct_stream stream);
ct_status ct_adjoint_backward(const ct_accel *accel, const ct_adjoint_desc *desc, const float *albedo,
                              const float *emission, const float *d_image, float *d_albedo, float *d_emission,
                              ct_stream stream);

/* ---------------------------------------------------------------------------
 * Neural radiance cache: a small fully fused MLP, bf16 weights with fp32
 * accumulation on the tensor cores (tcgen05.mma, accumulators in tensor
 * memory), queried with a path vertex to stand in for the radiance leaving
 * it (no counterpart in the reference).  Network: the 256-value encoding
 * below -> 5 hidden layers of 64 (ReLU, activations rounded to bf16) -> 16
 * outputs, the first three RGB.  Weights: one bf16 buffer of
 * CT_NRC_WEIGHT_COUNT values, row-major (output, input) per layer: W0
 * [64][256], W1..W4 [64][64], W5 [16][64]; 16-byte aligned device memory.
 * Encoding of a query (position, direction, normal, albedo), in order:
 *   position q = clamp((p - bbox_min) / bbox_extent, 0, 1); per axis c and
 *     band k < 16, t = (q_c 2^k) mod 2: sin(pi t), cos(pi t)   (96 values);
 *   direction and then normal, each as u0 = atan2(v.z, v.x) / 2pi + 1/2 and
 *     u1 = v.y / 2 + 1/2, one-blob encoded in 32 bins
 *     (exp(-((u - (i + 1/2) / 32) 32)^2 / 2), bin i)          (2 x 64 values);
 *   albedo (3 values); zeros up to 256.
 * ct_nrc_encode writes that encoding in bf16 ([n][256]); ct_nrc_infer runs
 * encoding and network on `n` queries and writes RGB (float[n][3]);
 * ct_nrc_infer_encoded runs the network on encoded inputs.  All pointers
 * are device memory.  ct_nrc_status reads (and with reset, clears) the
 * word a kernel sets when a tensor-core wait runs out (about one second;
 * the kernel then frees its tensor memory and returns). */
#define CT_NRC_INPUT_DIMS 256
#define CT_NRC_WIDTH 64
#define CT_NRC_HIDDEN_LAYERS 5
#define CT_NRC_OUTPUT_DIMS 16
#define CT_NRC_WEIGHT_COUNT (64 * 256 + 4 * 64 * 64 + 16 * 64)
typedef struct ct_nrc_query {
  float position[3];
  float direction[3];              /* unit vector */
  float normal[3];                 /* unit vector */
  float albedo[3];
} ct_nrc_query;                    /* 48 B */
typedef struct ct_nrc_net {
  uint64_t weights_address;        /* bf16[CT_NRC_WEIGHT_COUNT] */
  float bbox_min[3];
  float bbox_extent[3];            /* > 0 */
} ct_nrc_net;
ct_status ct_nrc_encode(const ct_nrc_net *net, const ct_nrc_query *queries, uint32_t n, void *encoded, ct_stream stream);
ct_status ct_nrc_infer(const ct_nrc_net *net, const ct_nrc_query *queries, uint32_t n, float *rgb, ct_stream stream);
ct_status ct_nrc_infer_encoded(const ct_nrc_net *net, const void *encoded, uint32_t n, float *rgb, ct_stream stream);
ct_status ct_nrc_status(int reset, uint32_t *out);

/* The path tracer of ct_adjoint_forward (one sample per pixel, seed
 * desc->seed, desc->miss_radiance), stopped at surface vertex v_c
 * (c = cache_vertex; v0 is the primary hit, so with the camera counted as
 * path vertex 0, v_c is path vertex c + 1), where the cache stands in for
 * the rest of the path:
 *   image = base + throughput * cache(query)
 * with base the radiance gathered at v0 .. v_{c-1} (their emission),
 * throughput a[v0] ... a[v_{c-1}], and query v_c's position, the direction
 * back along the ray, its normal and albedo.  Pixels whose path ends before
 * v_c get throughput 0 and a zero query.  Self-training paths: `train_paths`
 * pixels, the i-th at (train_offset + i * W * H / train_paths) mod (W * H),
 * trace the same path again past v_c for train_bounces more bounces; for
 * each of their vertices v_{c+j} (j < train_bounces) they record the query,
 * the radiance gathered from it up to the terminal vertex
 * v_{c+train_bounces}, and the throughput to it, and then the terminal
 * vertex's query, so that the caller's target is
 * partial + throughput * cache(terminal).  A training vertex that is not
 * reached has albedo -1 in its query.  All buffers are device memory; sizes
 * below. */
typedef struct ct_nrc_frame {
  uint32_t struct_size;            /* sizeof(ct_nrc_frame) */
  uint32_t train_paths;
  uint32_t train_offset;
  uint32_t train_bounces;          /* 1..8 */
  uint32_t cache_vertex;           /* 1..8 */
  uint32_t _reserved;              /* 0 */
  uint64_t base_address;           /* float[H*W][3] */
  uint64_t query_address;          /* ct_nrc_query[H*W] */
  uint64_t throughput_address;     /* float[H*W][3] */
  uint64_t train_query_address;    /* ct_nrc_query[train_paths][train_bounces + 1] */
  uint64_t train_partial_address;  /* float[train_paths][train_bounces][3] */
  uint64_t train_throughput_address; /* float[train_paths][train_bounces][3] */
} ct_nrc_frame;                    /* 72 B */
ct_status ct_nrc_trace(const ct_accel *accel, const ct_adjoint_desc *desc, const float *albedo,
                       const float *emission, const ct_nrc_frame *frame, ct_stream stream);

/* Reads (and with reset != 0 clears) the device status word.  Synchronises `stream`. */
ct_status ct_get_error(ct_stream stream, int reset, ct_error_info *out);

#ifdef __cplusplus
}
#endif

#ifdef __cplusplus
static_assert(sizeof(ct_aabb) == 24, "AABB");
static_assert(sizeof(ct_instance) == 72, "INSTANCE");
static_assert(sizeof(ct_primitive) == 8, "PRIMITIVE");
static_assert(sizeof(ct_material) == 84, "MATERIAL");
static_assert(sizeof(ct_light) == 40, "LIGHT");
static_assert(sizeof(ct_light_config) == 52, "LIGHT_CONFIG");
static_assert(sizeof(ct_reservoir) == 36, "RESERVOIR");
static_assert(sizeof(ct_path_reservoir) == 92, "PATH_RESERVOIR");
static_assert(sizeof(ct_velocity) == 8, "VELOCITY");
static_assert(sizeof(ct_di_info) == 60, "DIRECT_ILLUMINATION_INFO");
static_assert(sizeof(ct_camera_view) == 264, "camera_view");
static_assert(sizeof(ct_status_block) == 96, "Status");
static_assert(sizeof(ct_world) == 96, "WORLD");
static_assert(sizeof(ct_restir) == 72, "RESTIR");
static_assert(sizeof(ct_brush_config) == 28, "BRUSH_CONFIG");
static_assert(sizeof(ct_brush_counter) == 8, "BRUSH_COUNTER");
static_assert(sizeof(ct_push_constant) == 88, "PushConstant");
static_assert(sizeof(ct_ray_query) == 40, "ct_ray_query");
static_assert(sizeof(ct_ray_hit) == 16, "ct_ray_hit");
static_assert(sizeof(ct_adjoint_desc) == 72, "ct_adjoint_desc");
static_assert(sizeof(ct_params) == 128, "ct_params");
static_assert(sizeof(ct_view) == 224, "ct_view");
static_assert(sizeof(ct_nrc_query) == 48, "ct_nrc_query");
static_assert(sizeof(ct_nrc_net) == 32, "ct_nrc_net");
static_assert(sizeof(ct_nrc_frame) == 72, "ct_nrc_frame");
#endif

#endif /* CT_H */
