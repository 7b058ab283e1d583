/*
 * phox.h : C ABI of the B200 optical-photon engine (drop-in for the Opticks simulate path).
 *
 * All entry points return 0 on success and a negative code on failure; phx_last_error()
 * gives the message of the last failure on the calling thread.  No C++ exception crosses
 * this boundary.  Arrays are plain pointers with the Opticks byte layouts (see
 * opticks_b200/csrc/phx_pod.h).  One engine per device; calls on one engine are serialised
 * by the caller (the reference uses a process-wide singleton per GPU: QSim::INSTANCE,
 * CSGOptiX::INSTANCE).
 *
 * Reference interfaces replaced (paths within simoncblyth/opticks):
 *   phx_create            CSGOptiX::Create            CSGOptiX/CSGOptiX.cc:349
 *                         QSim::UploadComponents      qudarap/QSim.cc:119-262
 *                         CSGFoundry::upload          CSG/CSGFoundry.cc:3392
 *   phx_simulate          CSGOptiX::simulate(gs,eid)  CSGOptiX/CSGOptiX.cc:780
 *                         (python twin _CSGOptiXService.simulate  CSGOptiX/opticks_CSGOptiX.cc:24-110)
 *   phx_simulate_device   SSimulator::simulate_launch sysrap/SSimulator.h:16-37,
 *                         CSGOptiX::launch            CSGOptiX/CSGOptiX.cc:1091-1190
 *   phx_count_photons     SGenstep::GetNumPhoton / QEvt::setGenstepUpload  qudarap/QEvt.cc:199-330
 *   phx_csg_scan[_device] CSGScan / _CSGScan_intersect  CSG/CSGScan.cc:29-130, CSG/CSGScan.cu:11-25
 *   phx_rng_sequence      QSim::rng_sequence          qudarap/QSim.cc:1070-1168, qudarap/QSim.cu:43-68
 *   phx_trace[_device]    the trace step of simtrace  CSGOptiX/CSGOptiX7.cu:112-218, :563-603
 *   phx_simulate_batched  (no counterpart: the reference loops QSim::simulate per event,
 *                          qudarap/QSim.cc:436-595)
 *   phx_adjoint_device    (no counterpart: score-function gradients of expected hits)
 *   phx_destroy           CSGOptiX / QSim teardown
 */
#ifndef PHOX_H
#define PHOX_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct phx_engine phx_engine;

/* CSGFoundry arrays (CSG/CSGFoundry.cc:2978-3016 load) */
typedef struct {
    const float*   node;  int32_t num_node;   /* (num_node,4,4)  CSGNode  */
    const float*   prim;  int32_t num_prim;   /* (num_prim,4,4)  CSGPrim  */
    const int32_t* solid; int32_t num_solid;  /* (num_solid,3,4) CSGSolid */
    const float*   inst;  int32_t num_inst;   /* (num_inst,4,4)  qat4 instance transforms; the .w
                                                 column holds ins_idx, gas_idx, sensor_identifier+1,
                                                 sensor_index as int32 (sysrap/sqat4.h:345-389) */
    const float*   itra;  int32_t num_itra;   /* (num_itra,4,4)  inverse node transforms */
    const float*   plan;  int32_t num_plan;   /* (num_plan,4)    planes (convexpolyhedron) */
} phx_geometry;

/* SSim standard arrays: bnd (qudarap/QBnd.cc:130-165), optical (sysrap/sstandard.h:311-420),
 * scintillation inverse CDF (qudarap/QScint.cc:84-120) */
typedef struct {
    const float*    bnd;      int32_t num_bnd;  int32_t num_wl;   /* (num_bnd,4,2,num_wl,4) */
    float           wl_low;   float   wl_step;                    /* nm : 60, 1 */
    const uint32_t* optical;                                      /* (num_bnd*4,4) */
    const float*    icdf;     int32_t icdf_layers; int32_t icdf_width; int32_t hd_factor; /* (3,4096,1), 20 */
} phx_physics;

/* SEventConfig defaults (sysrap/SEventConfig.cc:40-110) */
typedef struct {
    uint64_t seed;                    /* curand_init seed                          0 */
    uint64_t offset;                  /* curand_init offset                        0 */
    uint64_t skipahead_event_offset;  /* OPTICKS_EVENT_SKIPAHEAD             100000 */
    int64_t  max_photon;              /* RNG state slots prepared at create  1000000 */
    int32_t  max_bounce;              /* OPTICKS_MAX_BOUNCE                       31 */
    float    max_time;                /* OPTICKS_MAX_TIME (ns)                 1e27 */
    float    propagate_epsilon;       /* OPTICKS_PROPAGATE_EPSILON (mm)        0.05 */
    float    propagate_epsilon0;      /* OPTICKS_PROPAGATE_EPSILON0 (mm)       0.05 */
    uint32_t epsilon0_mask;           /* OPTICKS_PROPAGATE_EPSILON0_MASK  TO,CK,SI,SC,RE */
    uint32_t hit_mask;                /* OPTICKS_HIT_MASK                          SD */
    int32_t  root_polish;             /* FP64 polish of quadratic leaf roots       0 */
    int32_t  num_sensor;              /* length of the per-sensor hit count output 0 */
    int32_t  kernel_mode;             /* 0: one thread per photon, 1: persistent threads with refill,
                                         2: wavefront rounds (closest hit and physics as separate kernels) */
    int32_t  block;                   /* persistent kernel block size (32, 64, 128, 256) */
    int32_t  regroup;                 /* persistent kernel: bounces between lane refills */
    int32_t  chunk;                   /* persistent kernel: queue grab per warp in units of 32 photons */
    int32_t  use_graph;               /* batched launches: capture once as a CUDA graph and replay */
    int64_t  wave_pool;               /* wavefront loop: in-flight path slots (180 B each); a call with
                                         more photons refills freed slots from its queue.  0 = every
                                         photon of the call in flight while that fits in half of the
                                         free device memory, at least 2^26 slots; the engine keeps its
                                         slots until phx_destroy (or phx_trim) */
    int32_t  wave_refill;             /* wavefront closest-hit kernel: idle lanes a warp waits for before
                                         it takes new rays (1..32; 12) */
    int32_t  wave_rounds;             /* wavefront schedule: n > 0 = n rounds and then the tail kernel
                                         for whatever is left, with no host read (a batched call is then
                                         captured as a CUDA graph, use_graph), when every photon of the
                                         call is in flight at once; 0, or a call that refills slots =
                                         the host reads the live count every few rounds and starts the
                                         tail kernel below wave_tail paths (2) */
    int64_t  wave_tail;               /* live paths at or below which the tail kernel finishes them
                                         (host-read schedule; 262144) */
    int32_t  adj_wave_rounds;         /* wave_rounds of phx_adjoint_device calls (12): its tail kernel
                                         carries the score terms and the tangent, so more bounces pay
                                         in the rounds than for plain calls */
} phx_config;

typedef struct {
    float*    photon;       /* (num_photon,4,4) sphoton, or NULL */
    uint64_t* seq;          /* (num_photon,2,2) seqhis[2],seqbnd[2], or NULL */
    float*    hit;          /* (hit_capacity,4,4) sphoton of selected photons in photon order, or NULL */
    int64_t   hit_capacity;
    uint32_t* sensor_hits;  /* (num_sensor) hits per sensor (identity-1), or NULL */
    int64_t   num_photon;   /* out */
    int64_t   num_hit;      /* out : hits selected (may exceed hit_capacity; then status has HIT_OVERFLOW) */
    uint32_t  status;       /* out : status bits: 0x1 CSG evaluator stack error, 0x2 traversal stack
                               overflow, 0x4 rejection-loop cap, 0x8 hit overflow, 0x10 photon index
                               beyond the prepared RNG states, 0x20 queue watchdog, 0x40 input photon
                               index beyond the input photon array */
} phx_outputs;

void        phx_config_default(phx_config* cfg);
const char* phx_last_error(void);
const char* phx_version(void);

int phx_create(const phx_geometry* geo, const phx_physics* phys, const phx_config* cfg, int device, phx_engine** out);
int phx_destroy(phx_engine* e);

/* Release the device memory the engine grew for its calls (no reference counterpart): the wavefront
 * path pool (180 B per in-flight path; by default every photon of the largest call), the event-advanced
 * RNG states, the host path's staging buffers and the hit-merge workspace.  For a host application
 * that shares the GPU after a large call; the next call allocates what it needs again.  Waits for
 * all work on the device first.  *bytes_released (optional) receives the bytes freed. */
int phx_trim(phx_engine* e, int64_t* bytes_released);

/* Change the launch shape of later calls (no reference counterpart): kernel_mode, block, regroup,
 * chunk, use_graph, wave_pool, wave_refill, wave_rounds, wave_tail and adj_wave_rounds are taken from *cfg (a smaller
 * wave_pool takes effect when the engine's pool is next released or grown), every other field is
 * ignored.  None of them changes results (every loop form gives the same photons, seq and hits);
 * they are the knobs the autotuner sets. */
int phx_set_launch_config(phx_engine* e, const phx_config* cfg);

/* sum of quad6 q0.w photon counts */
int64_t phx_count_photons(const float* gensteps, int32_t num_genstep);

/* host arrays in, host arrays out: gensteps (num_genstep,6,4) */
int phx_simulate(phx_engine* e, const float* gensteps, int32_t num_genstep, int32_t event_index, phx_outputs* out);

/* device arrays in and out (pointers in *out are device pointers); stream is a cudaStream_t or NULL.
 * num_photon must equal the sum of the genstep photon counts.  photon_offset is the absolute index of
 * the first photon (its RNG slot and sphoton.index), as params.photon_slot_offset of a genstep slice
 * launch (CSGOptiX/CSGOptiX7.cu:441); outputs still start at 0.  num_hit/status are returned to the host. */
int phx_simulate_device(phx_engine* e, const float* d_gensteps, int32_t num_genstep, int64_t num_photon,
                        int32_t event_index, int64_t photon_offset, phx_outputs* d_out, void* stream);

/* Allocation-free variant of phx_simulate_device.  No counterpart in the reference.
 * For callers that cannot allocate device memory per call (a framework whose caching allocator owns
 * all device memory, or a per-event loop that cannot take the device-wide synchronisation that
 * cudaMalloc/cudaFree may imply): it calls no cudaMalloc, cudaFree or allocating library routine.
 * Its scratch is one fixed device array in the library (about 2.6 MB, held on every GPU that loads
 * the library until the process exits), sized for at most 8,388,608 photons and 65,536 gensteps per
 * call; larger calls are rejected with an error.  Its bounce loop is always the one-kernel form
 * (the persistent work queue; one thread per photon with kernel_mode 0), never the wavefront rounds
 * that phx_simulate_device runs by default, because their path pool is sized per call: results are
 * bit-identical, throughput is that of kernel_mode 1.  Inputs and outputs are the caller's device
 * buffers as for phx_simulate_device; when hits or sensor counts are requested the photon output
 * must be given (hits are selected from it).  The photons must lie within the RNG slots prepared at
 * phx_create (config max_photon); otherwise the call is rejected rather than growing them.
 * The first call on a device looks up the device address of the scratch array (once per device);
 * make that first call before any stream capture.  The looked-up address is kept for the life of the
 * process: resetting the device (cudaDeviceReset) after the first call is not supported.  All calls share the one array: calls that
 * overlap on the GPU (on any engine of the same device) race; serialise them. */
int phx_simulate_device_noalloc(phx_engine* e, const float* d_gensteps, int32_t num_genstep, int64_t num_photon,
                                int32_t event_index, int64_t photon_offset, phx_outputs* d_out, void* stream);

/* Many events in one persistent launch (no reference counterpart: the reference loops
 * QSim::simulate per event, qudarap/QSim.cc:436-595).  gensteps (num_genstep,6,4) on device with
 * d_genstep_event[g] the event index of genstep g (non-decreasing).  Photon j of an event uses RNG slot j
 * advanced by skipahead(event * skipahead_event_offset), so every event's photons, seq and hits equal
 * those of phx_simulate_device for that event alone.  Outputs are the events' photons concatenated in
 * genstep order; hits are selected over the concatenation (in photon order).  block/chunk/regroup <= 0
 * take the engine config.  d_event_done_ns (num_event+1, optional) receives the %globaltimer value when
 * each event's last photon finished, and at [num_event] the launch start. */
int phx_simulate_batched_device(phx_engine* e, const float* d_gensteps, const int32_t* d_genstep_event,
                                int32_t num_genstep, int64_t num_photon, int32_t block, int32_t chunk,
                                int32_t regroup, int32_t num_event, uint64_t* d_event_done_ns,
                                phx_outputs* d_out, void* stream);

/* ray scan against one CSGPrim (CSGScan): rays SoA (6,n) = ox,oy,oz,dx,dy,dz ;
 * isect (n,4) = normal.xyz, t (t=0 for a miss) */
int phx_csg_scan(phx_engine* e, int32_t prim, float t_min, const float* rays, int64_t n, float* isect);
int phx_csg_scan_device(phx_engine* e, int32_t prim, float t_min, const float* d_rays, int64_t n, float* d_isect,
                        int32_t polish, void* stream);

/* Closest hit of arbitrary rays over the whole geometry: the trace step of simtrace
 * (CSGOptiX/CSGOptiX7.cu:563-603, which calls trace() :112-218 and records the PRD).  rays SoA (6,n) =
 * ox,oy,oz,dx,dy,dz ; prd (n,2,4) in the reference's quad2 layout (sysrap/squad.h:180-245):
 * q0 = world normal xyz (unnormalised, as the CH program leaves it), t ; q1 = lposcost, 0,
 * iindex<<16|identity, globalPrimIdx<<16|boundary, all of q1.zw 0xffffffff for a miss.  Hits with
 * t outside [t_min, t_max) are ignored.  *status (optional) receives the PHX_STATUS bits of the
 * rays (the call then synchronises the stream). */
int phx_trace(phx_engine* e, const float* rays, int64_t n, float t_min, float t_max, float* prd, uint32_t* status);
int phx_trace_device(phx_engine* e, const float* d_rays, int64_t n, float t_min, float t_max, float* d_prd, uint32_t* status,
                     void* stream);

/* per-photon uniform streams (QSim::rng_sequence): out (num_photon, num_per_photon) float32,
 * photon slots photon_offset..photon_offset+num_photon-1 advanced by the event skipahead */
int phx_rng_sequence(phx_engine* e, int32_t event_index, int64_t photon_offset, int64_t num_photon,
                     int32_t num_per_photon, float* out);

/* Score-function adjoint of the expected hits per sensor (no counterpart in the reference).
 * theta (HOST, 32 floats) = absorption length [0:8], Rayleigh length [8:16], reemission probability
 * [16:24] and refractive index [24:32] of the material of texture line mat_line (4*boundary+0 or +3),
 * piecewise constant in 8 bins of width (wl_hi-wl_lo)/8 over [wl_lo, wl_hi).  Every texture line of
 * that material is re-tabulated with theta for this call (the engine's own tables stay unchanged; the
 * group velocity in the bins is c/n).  One forward pass over the device gensteps accumulates
 * d_hits[s] = hits on sensor s and d_grad[s*32+k] = sum over those hits of d log p(path)/d theta_k
 * (absorption/scattering/sail densities, reemission and Fresnel branch probabilities).  With flags
 * PHX_ADJ_PATHWISE the refractive-index rows also carry the pathwise part: the refracted direction's
 * change with n, carried forward as a tangent of position, direction and polarisation into every
 * later segment length, incidence angle, Fresnel probability and Rayleigh density (the surface
 * curvature from a probe intersection of the hit prim); not carried: a tangent through a
 * reemission or a diffuse reflection (both redraw the direction), and hits that move across a
 * sensor's edge (the visibility boundary term).  d_hits, d_grad: device doubles, (num_sensor) and
 * (num_sensor*32); the engine must have config num_sensor > 0. */
#define PHX_ADJ_PATHWISE 0x1
int phx_adjoint_device(phx_engine* e, const float* d_gensteps, int32_t num_genstep, int64_t num_photon,
                       int32_t event_index, const float* theta, int32_t mat_line, float wl_lo, float wl_hi,
                       double* d_hits, double* d_grad, int32_t flags, void* stream);

/* Hit merging: SPM::merge_partial_select (sysrap/SPM.cu:110-200, called per launch from
 * QEvt::PerLaunchMerge qudarap/QEvt.cc:1172 and on concatenated results from QEvt::FinalMerge).
 * Records are sphoton (lite 0, 64 B) or sphotonlite (lite 1, 16 B).  Selects records with
 * (flagmask & select_flagmask) != 0 (0xffffffff: all records, already selected), groups them by the
 * key (identity << 48) | unsigned(time / time_window) and reduces each group to one record
 * (sphoton: the earliest record, flagmask OR, hitcount sum; sphotonlite: the first record, min time,
 * flagmask OR, hitcount sum: sysrap/sphoton.h:292-320, sysrap/sphotonlite.h:68-97).  Output is in
 * ascending key order.  time_window 0 returns the selected records in input order, unmerged.
 * *num_out receives the number of output records; when it exceeds out_capacity nothing is written
 * and the call fails (-3), so a caller can retry with *num_out (num_in rows are always enough).
 * The call synchronises the stream (the output count is read back), as the reference does.
 * num_in < 2^31.  Times are expected finite: a group whose times are all NaN keeps its first record. */
int phx_merge_hits_device(phx_engine* e, const void* d_in, int64_t num_in, int32_t lite, uint32_t select_flagmask,
                          float time_window, void* d_out, int64_t out_capacity, int64_t* num_out, void* stream);
/* host arrays in and out; same semantics */
int phx_merge_hits(phx_engine* e, const void* in, int64_t num_in, int32_t lite, uint32_t select_flagmask, float time_window,
                   void* out, int64_t out_capacity, int64_t* num_out);

/* Input photons (SEvt::setInputPhoton sysrap/SEvt.cc:602-640, uploaded as in qudarap/QEvt.cc:540-560):
 * a genstep of gencode 19 (OpticksGenstep_INPUT_PHOTON, numphoton N) makes each of its photons a
 * copy of photon[photon index] (sphoton rows, (num_photon,4,4) float32) with the TORCH flag set
 * (qudarap/qsim.h:2557); the photon index is the absolute one of phx_simulate_device.  An index
 * beyond num_photon leaves the photon zero and sets PHX_STATUS_INPUT_RANGE.  The host form copies
 * the array to the device; the device form uses the caller's buffer (16-byte aligned, kept alive
 * and unchanged while calls use it).  num_photon 0 clears.  Gencode 14 (CARRIER) needs no input. */
int phx_set_input_photon(phx_engine* e, const float* photon, int64_t num_photon);
int phx_set_input_photon_device(phx_engine* e, const float* d_photon, int64_t num_photon);

/* The black-body wavelength table (4096 floats, nm) that torch photons without a wavelength
 * sample (qudarap/qsim.h:2541-2544, QPlanck: 6500 K over 80-800 nm, qudarap/QPlanck.cc:36-48).
 * Host-only, no engine needed. */
int phx_planck_icdf(float* out, int n);

/* Diagnostics of the last phx_simulate / phx_simulate_device call on this engine (no reference
 * counterpart): kernels it launched and, in kernel_mode 2, wavefront rounds (one closest-hit and
 * one physics launch each) and, for phx_simulate_batched_device, whether it replayed a captured
 * CUDA graph (*graph 1). */
int phx_last_call_stats(phx_engine* e, int64_t* kernel_launches, int64_t* wave_rounds, int32_t* graph);

#ifdef __cplusplus
}
#endif
#endif
