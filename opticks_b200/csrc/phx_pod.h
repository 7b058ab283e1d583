// phx_pod.h : plain-old-data layouts shared by the host library and the device kernels.
//
// Every record here has the byte layout of the corresponding Opticks array so that
// arrays produced by the reference (CSGFoundry/*.npy, SSim standard bnd/optical/icdf,
// quad6 gensteps) can be handed over unchanged:
//
//   photon   64 B  sysrap/sphoton.h:171-260        (N,4,4) float32 view
//   seq      32 B  sysrap/sseq.h:54-65              (N,2,2) uint64  : seqhis[2], seqbnd[2]
//   genstep  96 B  sysrap/squad.h quad6             (G,6,4) float32 view
//   node     64 B  CSG/CSGNode.h:196                (Nn,4,4)
//   prim     64 B  CSG/CSGPrim.h:63-100             (Np,4,4)
//   inst     64 B  sysrap/sqat4.h:23-100            (Ni,4,4), identity ints in the .w column
//
// Flag values follow sysrap/OpticksPhoton.h:22-46, genstep codes sysrap/OpticksGenstep.h:21-42,
// CSG typecodes sysrap/OpticksCSG.h, torch types sysrap/storchtype.h:9-17,
// surface kinds ("ems") sysrap/smatsur.h:8-15.  They are file formats, so the numbers are the same.
#pragma once
#include <stdint.h>

// ---- photon history flags (one bit each; FFS gives the 4-bit seqhis nibble) ----
enum {
    PHX_CERENKOV           = 0x1 <<  0,
    PHX_SCINTILLATION      = 0x1 <<  1,
    PHX_TORCH              = 0x1 <<  2,
    PHX_BULK_ABSORB        = 0x1 <<  3,
    PHX_BULK_REEMIT        = 0x1 <<  4,
    PHX_BULK_SCATTER       = 0x1 <<  5,
    PHX_SURFACE_DETECT     = 0x1 <<  6,
    PHX_SURFACE_ABSORB     = 0x1 <<  7,
    PHX_SURFACE_DREFLECT   = 0x1 <<  8,
    PHX_SURFACE_SREFLECT   = 0x1 <<  9,
    PHX_BOUNDARY_REFLECT   = 0x1 << 10,
    PHX_BOUNDARY_TRANSMIT  = 0x1 << 11,
    PHX_NAN_ABORT          = 0x1 << 12,
    PHX_MISS               = 0x1 << 15
};

// ---- genstep codes (quad6 q0.i.x) ----
enum {
    PHX_GS_G4Cerenkov_1042         = 1,
    PHX_GS_G4Scintillation_1042    = 2,
    PHX_GS_DsG4Scintillation_r4695 = 5,
    PHX_GS_TORCH                   = 6,
    PHX_GS_CARRIER                 = 14,
    PHX_GS_CERENKOV                = 15,
    PHX_GS_SCINTILLATION           = 16,
    PHX_GS_G4Cerenkov_modified     = 18,
    PHX_GS_INPUT_PHOTON            = 19
};

// ---- torch source shapes (storch q5.u.w) ----
enum {
    PHX_T_UNDEF = 0,
    PHX_T_DISC,
    PHX_T_LINE,
    PHX_T_POINT,
    PHX_T_CIRCLE,
    PHX_T_RECTANGLE,
    PHX_T_SPHERE_MARSAGLIA,
    PHX_T_SPHERE,
    // extension with no reference counterpart: T_SPHERE directions with a random linear
    // polarisation perpendicular to the direction (one extra uniform, consumed last).
    PHX_T_SPHERE_RANDPOL = 64
};

// ---- event jump matrices of the XORWOW streams (phx_rngjump.h) ----
#define PHX_JUMP_BITS 160
#define PHX_JUMP_COLW 8                          // words per stored column (5 used)
#define PHX_JUMP_MATW (PHX_JUMP_BITS * PHX_JUMP_COLW)
// the same jump as XOR tables over 4-bit groups of the state: entry (g, k) = XOR of the columns
// 4g+b for the bits b set in k (40 groups x 16 patterns x PHX_JUMP_COLW words)
#define PHX_JUMP_NIBW (PHX_JUMP_BITS / 4 * 16 * PHX_JUMP_COLW)

#define PHX_PLANCK_N 4096                        // black-body wavelength ICDF entries (QPlanck)

// ---- CSG typecodes ----
enum {
    PHX_CSG_ZERO = 0,
    PHX_CSG_UNION = 1,
    PHX_CSG_INTERSECTION = 2,
    PHX_CSG_DIFFERENCE = 3,
    PHX_CSG_NODE = 11,
    PHX_CSG_CONTIGUOUS = 11,
    PHX_CSG_DISCONTIGUOUS = 12,
    PHX_CSG_OVERLAP = 13,
    PHX_CSG_LEAF = 101,
    PHX_CSG_SPHERE = 101,
    PHX_CSG_ZSPHERE = 103,
    PHX_CSG_CYLINDER = 105,
    PHX_CSG_BOX3 = 110,
    PHX_CSG_TORUS = 116,
    PHX_CSG_SLAB = 106,
    PHX_CSG_CONE = 108,
    PHX_CSG_CONVEXPOLYHEDRON = 112,
    PHX_CSG_DISC = 113,
    PHX_CSG_HYPERBOLOID = 117,
    PHX_CSG_INFCYLINDER = 119,
    PHX_CSG_PHICUT = 121,
    PHX_CSG_HALFSPACE = 125
};

// ---- surface kinds held in optical[line].y ----
enum {
    PHX_EMS_MATERIAL = 0,
    PHX_EMS_NOSURFACE = 1,
    PHX_EMS_SURFACE = 2,
    PHX_EMS_SURFACE_ZPLUS_SENSOR_A = 3,
    PHX_EMS_SURFACE_ZPLUS_SENSOR_CUSTOMART = 4
};

// ---- per-launch status bits returned through the C ABI ----
enum {
    PHX_STATUS_OK               = 0,
    PHX_STATUS_CSG_STACK        = 0x1 << 0,  // CSG evaluator stack/tranche error on some ray
    PHX_STATUS_BVH_STACK        = 0x1 << 1,  // traversal stack overflow (ray given up as a miss)
    PHX_STATUS_LOOP_CAP         = 0x1 << 2,  // a rejection loop hit its iteration cap
    PHX_STATUS_HIT_OVERFLOW     = 0x1 << 3,  // more hits than the hit buffer holds
    PHX_STATUS_RNG_RANGE        = 0x1 << 4,  // photon index beyond the prepared RNG states
    PHX_STATUS_QUEUE_WATCHDOG   = 0x1 << 5,  // persistent queue gave up
    PHX_STATUS_INPUT_RANGE      = 0x1 << 6   // INPUT_PHOTON genstep beyond the input photon array (photon left zero)
};

#define PHX_NSEQ 2
#define PHX_SEQ_SLOTS 32

typedef struct { float x, y, z, w; } phx_f4;

typedef struct {
    float pos[3]; float time;
    float mom[3]; uint32_t hitcount_iindex;
    float pol[3]; float wavelength;
    uint32_t orient_boundary_flag; uint32_t identity; uint32_t index; uint32_t flagmask;
} phx_photon;   // 64 B, sphoton

typedef struct { uint64_t seqhis[PHX_NSEQ]; uint64_t seqbnd[PHX_NSEQ]; } phx_seq;  // 32 B, sseq

// BVH leaf record : one (instance, CSGPrim) pair
typedef struct {
    int32_t  inst;          // index into the instance transform arrays
    int32_t  node_offset;   // root node of the prim's CSG tree
    uint32_t gp_bd;         // (globalPrimIdx & 0xffff) << 16 | (boundary & 0xffff)
    uint32_t ii_id;         // (iindex & 0xffff) << 16 | (identity & 0xffff), identity = sensor_id+1
} phx_leaf;

// wide (4-ary) BVH node, child boxes stored per axis so one 128 B node is two sectors
typedef struct {
    float lo_x[4], hi_x[4], lo_y[4], hi_y[4], lo_z[4], hi_z[4];
    int32_t child[4];   // >=0 : inner node ; <0 : leaf range  -(1 + (first << 3 | (count-1)))
    int32_t pad[4];
} phx_bvh4_node;
