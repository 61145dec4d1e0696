/* exact-ballpark-b200: the C ABI of the batched destiny tick on sm_100a.
 *
 * Plain C: pointers and sizes, no torch types. Every entry point launches on the caller's CUDA stream, allocates
 * nothing and never synchronises the host, so a caller may capture it in a CUDA graph. Return codes: 0 success;
 * EBB_EINVAL (-1) for refused arguments (nothing launched); a positive value is a cudaError_t from the launch
 * (ebb_error_string names it). Device-side domain problems are reported through the status word some calls take.
 *
 * The flight-mode park's state is structure-of-arrays in device memory: a vector field is 3 (or 4) consecutive
 * planes of n values (x plane, y plane, z plane); Destiny's float members are stored as float, its doubles as
 * double. The reference keeps the same state as [n, 3] float64 tensors (exact_ballpark/vec_modes_cuda.py:280-290).
 */
#ifndef EBB_H
#define EBB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EBB_ABI_VERSION 8
#define EBB_EINVAL (-1)
#define EBB_ETOOBIG (-2)

/* The allocation-free tick's limits: rows its fixed records buffer holds, and devices it keeps an address for. */
#define EBB_NOALLOC_MAX_ROWS 262144
#define EBB_NOALLOC_MAX_DEVICES 64

/* The flight-mode park (one row a ship; rows grouped in worlds by the caller), field for field the state the
 * reference's xbpm_tick reads and writes (exact_ballpark/vec_modes_cuda.cu:83-96), laid out as above. */
typedef struct EbbFlightState {
    int64_t n;
    double friction, dt;          /* k and the tick in seconds */
    float ffriction, fdt;         /* the same as C floats */
    int32_t new_orbit;            /* Destiny's process-global useNewOrbit */
    int32_t dynamical;            /* dynamical orientation on */
    double *pos, *vel, *old_pos, *old_vel, *goto_pt, *last_g;   /* [3][n] */
    double *mass, *time_factor, *last_collision;               /* [n] */
    float *radius, *max_vel, *agility, *speed_fraction, *follow_range, *max_ang_vel, *rot_agility, *rot_roll;
    float *rot, *old_rot;                                      /* [4][n] x, y, z, w */
    float *ang_vel, *old_ang_vel, *torque;                     /* [3][n] */
    int64_t *ids, *effect_stamp, *follow_id, *owner_id, *clock;
    int32_t *mode, *follow_ptr;                                /* follow_ptr: the target's row, -1 for none */
    uint8_t *free_, *moribund, *massive, *interactive, *sensor;
} EbbFlightState;

/* The collision park (the gradient method on spheres): W worlds of N ball slots, world w is slots [w N, (w + 1) N),
 * each world's balls in its first slots in ascending id (an empty slot has exists = 0). The layout is the
 * reference's [W, N] tensors, row-major: a vector field is [W N][3] (x, y, z of a slot together), the collision list
 * [W N][hit_cap] (hit_cap = 3 (N - 1), at least 1), the impact record [W N][impact_cap] (impact_cap = N - 1, at least
 * 1). Field for field the state of exact_ballpark.vec_collide.VecCollidePark (vec_collide.py:470-512). */
#define EBB_COLLIDE_MAX_SLOTS 64
#define EBB_COLLIDE_MAX_STATICS 64
typedef struct EbbCollideState {
    int64_t worlds, slots, hit_cap, impact_cap;
    double friction, dt;
    double *pos, *vel, *old_pos, *old_vel, *goto_pt, *last_g, *last_c;                 /* [W N][3] */
    double *mass, *radius, *max_vel, *agility, *speed_fraction, *time_factor, *last_collision;   /* [W N] */
    int64_t *id, *mode, *level, *key, *mod;                                            /* key, mod [W N][3] */
    uint8_t *exists, *free_, *massive, *junk, *cloaked;
    int64_t *hits, *hits_n;                                                            /* [W N][hit_cap], [W N] */
    int64_t *imp_slot, *imp_n;                                                         /* [W N][impact_cap], [W N] */
    double *imp_s, *imp_closing;                                                       /* [W N][impact_cap] */
    /* static collidables (capsules, oriented boxes): S slots a world (0: none; at most EBB_COLLIDE_MAX_STATICS), each
     * a record of 175 doubles and 5 integers (kind, id, parent id, level, boxes) and up to B box keys, made once at the
     * load (exact_ballpark_b200.statics; vec_collide.py:261); hit_cap then counts S more entries */
    int64_t statics, boxes;
    uint8_t* s_exists;                                                                 /* [W S] */
    double* s_geo;                                                                     /* [W S][175] */
    int64_t *s_int, *s_keys;                                                           /* [W S][5], [W S][B][3] */
} EbbCollideState;

/* The combat park (missiles, formations, cloaking; exact_ballpark.vec_combat.VecCombatPark, vec_combat_cuda.cu:53-74):
 * the flight park's rows and, per row, whether it holds a ball (an empty row is moribund and inert until AddBall),
 * the leader's formation (char semantics, -1 none) and slot bits, a missile's owner row (-1 none), the tick's
 * contact and dispatch counts, and the bubble and cloak the commands keep; the formation table [formations][max
 * slots][3] with each formation's length. Dynamical orientation is required (flight.dynamical = 1). */
typedef struct EbbCombatState {
    EbbFlightState flight;
    uint8_t* exists;
    int64_t *formation_id, *formation_slots, *owner_ptr;
    int64_t *hits_n, *ev_n;                    /* out: contacts with the target this tick; target collisions dispatched */
    uint8_t* ev_self;                          /* out: the master's self-collision dispatched */
    int64_t *bubble, *cloaked, *flags;
    const double* formations;
    const int64_t* formation_len;
    int64_t n_formations, max_slots, tick_ms;
    int32_t do_missiles_off, master;
    const uint8_t* active;                     /* OnTick's per-world mask ([n] bytes, a world's rows alike), or null */
} EbbCombatState;

/* The composed park (exact_ballpark.vec_composed.VecComposedPark: the combat park with the gradient method's collisions
 * between every massive ball, missiles included): the combat state and, per row, its world label (a world's rows are
 * contiguous), the collision acceleration mLastC [3][n], the partition's filing (level [n], key and adjacent side
 * [3][n]) and the collision list [n][hit_cap] (hit_cap = 3 (S - 1) + 1 for worlds of at most S rows: three appends a
 * candidate and the master's self-collision). */
#define EBB_COMPOSED_FLAG_WARP_MASSIVE 64
#define EBB_COMPOSED_FLAG_PARTITION 128
typedef struct EbbComposedState {
    EbbCombatState combat;
    const int64_t* world;
    double* last_c;
    int64_t *level, *key, *mod, *hits;
    int64_t hit_cap;
} EbbComposedState;

/* The server layer over the flight park (exact_ballpark.vec_server.VecServer with its ModesAdapter): W worlds of one
 * bubble, each world's rows listed in the order its balls were added ([W][width], -1 padded) with their Destiny ids
 * (0 padded); per row its pilot (-1 none), the adapter's exists byte and the park's host-side columns (world label,
 * cloak, bubble, the re-filing count); the layer's own state per world (the next stamp, the bubble update's park time,
 * a dead bubble seen at an evolve) and per row (the old bubble settled, the last additions' fresh and listed flags).
 * A queued call's kind is its event's code, the index of the event's name in the reference's KINDS table
 * (vec_server.py:118-123). */
enum {
    EBB_KIND_GOTO_POINT = 1, EBB_KIND_GOTO_DIRECTION, EBB_KIND_STOP, EBB_KIND_FOLLOW_BALL, EBB_KIND_ORBIT,
    EBB_KIND_WARP_TO, EBB_KIND_ENTITY_WARP_IN, EBB_KIND_SET_SPEED_FRACTION, EBB_KIND_SET_MAX_SPEED, EBB_KIND_SET_MASS,
    EBB_KIND_SET_AGILITY, EBB_KIND_SET_RADIUS, EBB_KIND_SET_VELOCITY, EBB_KIND_SET_MASSIVE, EBB_KIND_SET_INTERACTIVE,
    EBB_KIND_SET_POSITION, EBB_KIND_CLOAK, EBB_KIND_UNCLOAK, EBB_KIND_SET_MAX_ANGULAR_SPEED,
    EBB_KIND_SET_ANGULAR_VELOCITY, EBB_KIND_SET_ROTATION, EBB_KIND_SET_ANGULAR_AGILITY,
    EBB_KIND_SET_MAX_ANGULAR_VELOCITY, EBB_KIND_LAUNCH_MISSILE, EBB_KIND_SET_TROLL, EBB_KIND_SET_FREE
};
enum { EBB_ROUTE_NONE = 0, EBB_ROUTE_BUBBLE = 1, EBB_ROUTE_CHARACTER = 2 };
#define EBB_SERVER_MAX_SLOTS 256
typedef struct EbbServerState {
    EbbFlightState flight;
    int64_t worlds, width;
    const int64_t *world_rows, *world_ids;     /* [W][width] */
    const int64_t* pilot;                      /* [n] */
    const uint8_t* exists;                     /* [n] */
    const int64_t* label;                      /* [n] the park's world label */
    int64_t *cloaked, *bubble, *refiled;       /* [n] */
    int64_t *stamp_for_system, *bubble_time;   /* [W] */
    uint8_t* dead;                             /* [W] */
    uint8_t *settled, *fresh, *listed;         /* [n] */
    double neg_kdt;                            /* -friction x dt: the decay factor's numerator */
    int32_t master;
} EbbServerState;

/* One tick's queue: J slots (the pushes, in order), each a kind [J] and per world its pushed byte (bit 0 pushed; bit
 * 1 the call already tested by an undo of a pending cloak, bit 0 then its queued flag and the local argument
 * CloakBall's tested bubble: no duplicate test again; the tested calls are a prefix of the queue), ball id, target id,
 * float arguments (4), int argument and SetBallPosition's local flag ([J][W], f [J][W][4]); out: per slot and world the
 * queued flag, the ball's and target's rows (-1 none) and the local argument or CloakBall's bubble (0, or -1 before
 * the ball's old bubble is its bubble) ([J][W]); the routes [J][W]; the uncloaks' AddBallsToPark recipients [J][n]
 * (rows of other slots untouched); the world's stamp and park time [W]; the send flags [n]. */
typedef struct EbbServerQueue {
    int64_t slots;
    const int32_t* kinds;
    const uint8_t* mask;
    const int64_t *ball, *target, *n, *loc_in;
    const double* f;
    uint8_t* ok;
    int64_t *row, *trow, *loc;
    int8_t* route;
    uint8_t* notice;
    int64_t *stamp, *clock;
    uint8_t *has_character, *gets_bubble;
} EbbServerQueue;

/* The master's partition and bubble partition over a flight park's rows (exact_ballpark.vec_space.VecSpace's
 * layer, vec_space.py:777; this build's slice: each ball's filing, the partition's boxes with BoxAllocator's kept
 * count, the top boxes' bubbles, the bubble dictionaries, the interactive and keep-alive sets, InitializeBubbles,
 * CopyBubbles, the tick's dead-bubble flags and re-filings). W worlds of N slots (N at most EBB_SPACE_MAX_SLOTS);
 * `rows` maps a slot to its park row (-1 for none). Every per-slot array is [N][W], every per-entry array [cap][W]
 * and every key [3][cap][W] (world w's entry e at e W + w), one thread a world; or, with `pitch` > 0, world-major:
 * each pointer names world 0's copy of its array, entries consecutive in the shapes below without their [W], and world
 * w's copy of every array starts w `pitch` bytes further on (`rnd` excepted: [W][EBB_RAND_WORDS] in both
 * arrangements); there the box table's per-entry fields (box_level, box_key's three, box_balls, box_kids,
 * box_bubble, box_parent, box_top, box_home, box_slot) are records of EBB_SPACE_BOX_RECORD words an entry, at words
 * 0, 1-3, 4, 5, 6, 7, 8, 9 and 10, each field's pointer naming it in world 0's entry 0. Capacities a world: `boxes` box-table
 * entries (and the same for the fill's stack), `dicts` bubble dictionaries, `entries` dictionary entries in insertion
 * order, `sets` members of the interactive sets and of the keep-alive sets. A world that leaves the layer's domain is
 * flagged (EBB_SPACE_FLAG_*) and left alone by later operations. Field for field the state the reference's layer keeps
 * in its `st` tensors (vec_space.py:808-830), with a box table in place of its top-box table. */
#define EBB_SPACE_MAX_SLOTS 128
#define EBB_SPACE_BOX_RECORD 16   /* words a box-table entry's record (world-major: one 128-byte line an entry) */
enum {  /* the tape's operations, numbered as the reference's OPS (vec_space.py:159) */
    EBB_SPACE_NONE = 0, EBB_SPACE_ADD = 1, EBB_SPACE_REFILE = 2, EBB_SPACE_INIT_BUBBLES = 3,
    EBB_SPACE_COPY_BUBBLES = 4, EBB_SPACE_KEEP_ALIVE = 5, EBB_SPACE_SET_INTERACTIVE = 6, EBB_SPACE_ADD_SENSOR = 7,
    EBB_SPACE_REMOVE_SENSOR = 8, EBB_SPACE_NOTIFY_RANGE = 9, EBB_SPACE_TRACK = 10, EBB_SPACE_REMOVE_BALL = 11,
    EBB_SPACE_DEAD = 12, EBB_SPACE_AFTER_EVOLVE = 13, EBB_SPACE_CLEAR_EVENTS = 14,
    /* this build's own, no number in the reference's OPS: HandleProximities alone (the reference runs it inside
     * AFTER_EVOLVE, as this one does) and the cloak attribute a sensor's candidates and CheckVisibility read */
    EBB_SPACE_HANDLE_PROXIMITIES = 18, EBB_SPACE_SET_CLOAKED = 19
};
enum {  /* an event's kind (the reference's EVENTS, vec_space.py:164) */
    EBB_SPACE_EV_PROXIMITY = 1, EBB_SPACE_EV_RANGE = 2, EBB_SPACE_EV_TRACKING = 3
};
enum {  /* a world's flags, the reference's FLAG bits (vec_space.py:171) and UNDEFINED (a deleted box read) */
    EBB_SPACE_FLAG_EVENTS = 1, EBB_SPACE_FLAG_TOPS = 2, EBB_SPACE_FLAG_EDGE = 4, EBB_SPACE_FLAG_BOXES = 8,
    EBB_SPACE_FLAG_DICTS = 16, EBB_SPACE_FLAG_ENTRIES = 32, EBB_SPACE_FLAG_PROXIMITY = 64,
    EBB_SPACE_FLAG_SENSOR_LIST = 128, EBB_SPACE_FLAG_HUGE = 256, EBB_SPACE_FLAG_BAD_OP = 512,
    EBB_SPACE_FLAG_SETS = 1024, EBB_SPACE_FLAG_UNDEFINED = 2048
};
typedef struct EbbSpaceState {
    int64_t worlds, slots, boxes, dicts, entries, sets;
    const int64_t* rows;                                          /* [N][W] */
    int64_t *level, *key, *mod, *active, *bubble, *old_bubble, *seq;   /* [N][W]; key, mod [3][N][W] */
    int64_t *my_box, *my_top;          /* [N][W] the box-table entries of a filed ball's box and of its top box */
    uint8_t *in_park, *keep_alive, *dead, *dropped;                /* [N][W] */
    int64_t *box_level, *box_key, *box_balls, *box_kids, *box_bubble, *stack;   /* [boxes][W]; key [3][boxes][W] */
    int64_t *box_n, *free_boxes;                                   /* [W] */
    int64_t *box_hash;              /* [2 boxes][W] the table's index: entry + 1 by (level, key), linear probing */
    int64_t *box_free, *box_free_n;                                /* [boxes][W] the free entries, [W] their count */
    int64_t *dict_bubble, *dict_n;                                 /* [dicts][W], [W] */
    int64_t *entry_bubble, *entry_id, *entry_value, *entry_n;      /* [entries][W], [W] */
    int64_t *inter_bubble, *inter_id, *inter_n;                    /* [sets][W], [W] */
    int64_t *keep_bubble, *keep_id, *keep_n;                       /* [sets][W], [W] */
    int64_t *bubble_id, *seq_next, *flags;                         /* [W] */
    /* The proximity sensors, notification ranges and target tracking (space.py:1345-1523; the reference's layer keeps
     * them in its srange ... pmap tensors, vec_space.py:825-836). Per slot [N][W]: the sensor's range (a float's
     * value), period and elapsed time, its only-interactives flag, the ball's proximity flag, its notification range
     * and in-range flag, its tracked slot (-1 none) with the range and in-range flag, the cloak attribute. A sensor's
     * balls and the world's proximity balls are std::unordered_maps whose iteration order is kept as libstdc++ keeps
     * it: their keys (slots) in that order, [cap][N][W] and [cap][W] (cap = `umap_cap` keys, at most
     * EBB_SPACE_MAX_SLOTS), each with its length and bucket count (1 for a fresh map). Events [events][W], each an
     * int32: kind | value << 4 | ball slot << 8 | other slot << 16, their count [W] (past `events`, counted, dropped
     * and the world flagged EVENTS). `rnd` [W][EBB_RAND_WORDS]: each world's glibc rand() state (ebb_glibc_srand),
     * drawn by a shuffled sensor. */
    int64_t umap_cap, events;
    double *srange, *speriod, *selapsed, *ntf_range, *trk_range;   /* [N][W] */
    int64_t *trk, *cloaked;                                        /* [N][W] */
    uint8_t *sonly, *has_prox, *ntf_in, *trk_in;                   /* [N][W] */
    uint8_t* slist;                                                /* [umap_cap][N][W] */
    int32_t *slen, *sbkt;                                          /* [N][W] */
    uint8_t* pmap;                                                 /* [umap_cap][W] */
    int32_t *pn, *pbkt;                                            /* [W] */
    int32_t* ev;                                                   /* [events][W] */
    int64_t* evn;                                                  /* [W] */
    int32_t* rnd;                                                  /* [W][EBB_RAND_WORDS] */
    uint64_t *smask, *pmask;   /* the same keys as sets of slots (128 bits): [2][N][W] a sensor's, [2][W] the map's */
    int64_t lanes;             /* 1: a thread runs a world; 32: a warp runs a world (GetNearbyBalls split over it) */
    int64_t pitch;             /* 0: the [..][W] arrangement; > 0 (a multiple of 16): world-major, bytes a world */
    int64_t *box_parent, *box_top;   /* [boxes][W] a box's parent entry (-1 for a top box), its top box's entry */
    int64_t *box_home, *box_slot;    /* [boxes][W] a box's home slot in box_hash, and the slot it sits in */
    int64_t* fbox;     /* [8][N][W] a filed ball's box entries by side (bit c: the box beside its own on axis c) */
} EbbSpaceState;
/* K operations a world, applied in order: code, a (a slot), b (an integer argument), each [K][W], and f, each
 * operation's floating-point arguments [K][4][W] (ADD_SENSOR: range, period; NOTIFY_RANGE: range; TRACK: range, and
 * f[1] nonzero when the target's id is 0, which turns tracking off; b: ADD_SENSOR's flags, bit 0 only interactives,
 * bit 1 shuffled; TRACK's target slot, -1 when the target is not a ball of the world; SET_CLOAKED's value). */
typedef struct EbbSpaceTape {
    int64_t K;
    const int64_t *code, *a, *b;
    const double* f;
} EbbSpaceTape;
/* One query a world over the layer's state (the reference's QUERIES, vec_space.py:160, and its xbps_query_*): kind,
 * a [W] (a slot), b [W] (a slot or flags), f [5][W]; out [1 + N][W]: out[0] the answer (VISIBILITY: the occluding
 * ball's id, 0 none, -2 between bubbles; RANGE_BALL, RANGE_POINT, NEARBY: the count of balls, -1 when the reference
 * ball is none of the world's; BUBBLE_AT: the bubble, -2 for no top box), out[1 + i] the balls' ids in order; outd
 * [N][W] their squared distances (RANGE_*). VISIBILITY: a source, b destination (-1: not a ball); RANGE_BALL: a the
 * ball, f[0] the range, b bit 0 cloaked balls too; RANGE_POINT: f[0..2] the point, f[3] the range, b as RANGE_BALL;
 * BUBBLE_AT: f[0..2]; NEARBY (GetNearbyBalls): a the ball, b bit 0 exclude fixed, bit 1 exclude inert, bit 2 exclude
 * cloaked. */
enum { EBB_SPACE_Q_VISIBILITY = 1, EBB_SPACE_Q_RANGE_BALL = 2, EBB_SPACE_Q_RANGE_POINT = 3, EBB_SPACE_Q_BUBBLE_AT = 4,
       EBB_SPACE_Q_NEARBY = 5 };
typedef struct EbbSpaceQuery {
    int64_t kind;
    const int64_t *a, *b;
    const double* f;
    int64_t* out;
    double* outd;
} EbbSpaceQuery;

/* The ABI version (EBB_ABI_VERSION). Replaces xbpm_abi / xbpo_abi (exact_ballpark/vec_modes_cuda.cu:750,
 * vec_orient_cuda.cu:499). */
int ebb_abi(void);

/* A cudaError_t's name, for a positive return code. Replaces xbpo_error_string (vec_orient_cuda.cu:503). */
const char* ebb_error_string(int code);

/* Bytes of device scratch ebb_flight_tick needs for n rows (the prepass's records). */
int64_t ebb_flight_scratch_bytes(int64_t n);

/* One tick of every world of the park in place: the prepass (each ship's start-of-tick position and velocity, its
 * vertical velocity after its own turn, whether it starts warp proper) into `scratch`, then each ship's tick (phase 1,
 * phase 3, phase 4, PetrifyTroll, its world's clock), one thread a ship. `scratch` holds at least
 * ebb_flight_scratch_bytes(n) bytes of device memory, 256-byte aligned; block is a multiple of 32 up to 256.
 * Replaces xbpm_tick (exact_ballpark/vec_modes_cuda.cu:754), which exact_ballpark.vec_modes_cuda.tick calls
 * (vec_modes_cuda.py:322). */
int ebb_flight_tick(const EbbFlightState* s, void* scratch, int64_t scratch_bytes, void* stream, int block);

/* ebb_flight_tick without caller scratch, for callers that cannot allocate device memory: an engine whose own
 * allocator owns the GPU's memory and hands none out, a loop that must not allocate once it runs, or a binding from a
 * language with no CUDA allocator at hand. The records go to a fixed buffer inside the library (EBB_NOALLOC_MAX_ROWS
 * rows, about 14.4 MB of device memory on every device that loads the library, held until the process exits), so
 * parks of more rows are refused with EBB_ETOOBIG, nothing launched. The same kernels and results as ebb_flight_tick.
 * The first call on a device looks up the buffer's device address (cudaGetSymbolAddress, with that device current);
 * make that first call before any stream capture. The address is kept for the life of the process, so a device reset
 * (cudaDeviceReset) or a new primary context on that device after the first call is not supported: the kept address
 * would name the old context's memory. `block` is a multiple of 32 up to 256, as for ebb_flight_tick. All calls on a
 * device share the buffer: calls that may overlap on the GPU (other streams, other threads) race on it and must be
 * ordered by the caller. Each call writes every record it reads, so the buffer needs no clearing. No counterpart in
 * the reference. */
int ebb_flight_tick_noalloc(const EbbFlightState* s, void* stream, int block);

/* The same tick with the worlds packed into tiles, one thread block a tile, the prepass's records in shared memory
 * (no scratch, one launch): tile_rows[0..tiles] are row offsets, each tile a run of whole worlds of at most
 * `tile_cap` rows (<= 4096), rows of a world contiguous; `block` threads (a multiple of 32, <= 256) take the tile's
 * ships 32 to a warp. status[0] is set nonzero if a follow_ptr leaves its tile (the ship is then ticked without its
 * target, as a missing target). The grid is persistent: `grid` blocks take tiles in turn. The tile size, block and
 * grid are the autotuner's choice (exact_ballpark_b200.autotune). No counterpart in the reference (its tick is two
 * launches, xbpm_tick). */
int ebb_flight_tick_tiled(const EbbFlightState* s, const int64_t* tile_rows, int64_t tiles, int tile_cap,
                          int32_t* status, void* stream, int block, int grid);

/* Rows a tile of ebb_flight_tick_worlds holds at most. */
#define EBB_WORLDS_MAX_TILE 1024

/* One tick of a list of worlds, each a contiguous run of rows anywhere in the park (a serving loop's resident
 * episodes, or the worlds with a tick under OnTick's mask): world w is rows [worlds[2w], worlds[2w + 1]), worlds never
 * overlap; tile t is the worlds [tile_worlds[t], tile_worlds[t + 1]), at most `tile_cap` rows (<= EBB_WORLDS_MAX_TILE)
 * and `tile_cap` worlds, gathered into one thread block's shared memory with their records; `grid` persistent blocks
 * take the `tiles` tiles in turn. Rows of no listed world are neither read nor written. With `active` [n] non-null,
 * rows whose byte is 0 keep their state bit for bit and the others tick as in the unmasked tick (OnTick's mask inside
 * the kernel, in place of a save and put-back of every row). status[0] bits: 1 a follow pointer leaving its world
 * (ticked without its target), 2 a malformed tile (skipped). Replaces the masked tick of
 * exact_ballpark.vec_orient.masked_tick (vec_orient.py:217) over xbpm_tick (vec_modes_cuda.cu:754); the listing
 * of worlds has no counterpart in the reference. */
int ebb_flight_tick_worlds(const EbbFlightState* s, const int64_t* worlds, const int64_t* tile_worlds, int64_t tiles,
                           int tile_cap, const uint8_t* active, int32_t* status, void* stream, int block, int grid);

/* Host-side planning for ebb_flight_tick_worlds: packs `count` worlds (rows [starts[k], starts[k] + lens[k]), each of
 * at most tile_cap rows; empty ones left out) into tiles of at most tile_cap rows, best-fit decreasing (the tiles
 * need not be runs of adjacent worlds), each tile's worlds in row order. Writes worlds[2 x listed] and
 * tile_worlds[tiles + 1] (caller arrays of 2 x count and count + 1 entries) and returns the number of tiles, or
 * EBB_EINVAL. No device work. No counterpart in the reference. */
int64_t ebb_plan_worlds(const int64_t* starts, const int64_t* lens, int64_t count, int tile_cap, int64_t* worlds,
                        int64_t* tile_worlds);

/* Rows copied between two parks, every field: src row src_rows[k] into dst row dst_rows[k], k < m (device arrays).
 * A follow pointer moves with its row, so a world moved as one run keeps its targets; a pointer that would leave dst
 * becomes -1, and rows outside either park are skipped (status[0] bit 4 for both). Admission and retirement of a
 * serving loop's episodes. No counterpart in the reference (its parks are loaded whole). */
int ebb_flight_move(const EbbFlightState* dst, const EbbFlightState* src, const int64_t* src_rows,
                    const int64_t* dst_rows, int64_t m, int32_t* status, void* stream, int block);

/* One tick of the collision park in place (TIME-706/707): the free balls' behaviours (GOTO's thrust, STOP's
 * damping), Gradient for every free massive ball (Potential with each collision candidate in Partition::
 * GetNearbyBalls' order, the overlap recursion, the impact and overlap responses, the later impact kept; then its
 * static collidables in the walk's order, CollideWithBall and ReactToCollision, COL-712), the commit and
 * the re-filing of the balls that moved. `active` [W] (nullable): only those worlds tick. One launch, one thread block
 * a group of whole worlds (N <= EBB_COLLIDE_MAX_SLOTS). status[0] bit 2: a re-filing at the grid's edge. Replaces
 * VecCollidePark.evolve's gradient path (exact_ballpark/vec_collide.py:990) and its kernels xbpc_tick / xbpc_gradient
 * (vec_collide_cuda.cu:1312-1530). */
int ebb_collide_tick(const EbbCollideState* s, const uint8_t* active, int32_t* status, void* stream);

/* The load's device steps for every existing slot (the host has written AddBall's clamped values): the decay factor
 * exp(-k dt / m) with glibc's exp (0 for m <= 0) and the first filing. status[0] bit 1: a filing the reference refuses
 * (a key at the grid's edge, or a ball wider than a top box). Replaces VecCollidePark.load's time factor and
 * _filing / _check_filing (vec_collide.py:550-667, 776-807). */
int ebb_collide_load(const EbbCollideState* s, int32_t* status, void* stream);

/* One tick of the combat park in place, in tiles of whole worlds (tile_rows[tiles + 1], each tile at most `block`
 * rows, one block a tile): the records pass, phase 1 for every ball (the releases by a target starting warp proper,
 * each mode's thrust with MISSILE and FORMATION, dynamical orientation unless disabled for missiles), each massive
 * normal missile's contacts with its target (Potential's recursion, counted), then phases 3 and 4 (the warp path or
 * the integrator, the rotation a tick on or a disabled missile's snap, the commit, the dispatch counts, PetrifyTroll,
 * the clock), block barriers between the steps. status[0] bit 0: a follow target outside its tile; bit 1: a tile
 * wider than the block. Replaces xbpc_tick (exact_ballpark/vec_combat_cuda.cu:731-800: its prepass, phase-1, contact
 * and commit launches), which exact_ballpark.vec_combat_cuda.tick calls (vec_combat_cuda.py:289). */
int ebb_combat_tick(const EbbCombatState* s, const int64_t* tile_rows, int64_t tiles, int32_t* status, void* stream,
                    int block);

/* One tick of the composed park in place, in tiles of whole worlds as ebb_combat_tick: the records pass, phase 1 (the
 * live balls' collision lists cleared), the warp paths with the drop-outs (re-filed at rest), the gradient for every
 * live massive ball in its world (GetNearbyBalls' candidates in the partition's walk order with a normal missile's
 * target its one candidate, Potential's recursion, COL-711's missile exception, the later-impact rule, the collision
 * list), then phases 3 and 4 with mLastG + mLastC, the re-filing of the balls that moved, the dispatch and the
 * master's self-collision appended; flags FLAG_WARP_MASSIVE and FLAG_PARTITION on the rows. Replaces
 * xbpp_tick (exact_ballpark/vec_composed_cuda.cu:421-509: its thirteen launches), which
 * exact_ballpark.vec_composed_cuda.tick calls. */
int ebb_composed_tick(const EbbComposedState* s, const int64_t* tile_rows, int64_t tiles, int32_t* status,
                      void* stream, int block);

/* Ball::InsertInBoxes' outcome (level, key, adjacent side) for the rows in `mask` ([n] bytes), from each row's state
 * or the given position, velocity ([3][n] planes) and speed fraction ([n] floats), any of them null for the row's
 * own; a filing the reference refuses (a key at the grid's edge, a ball wider than a top box) raises
 * EBB_COMPOSED_FLAG_PARTITION on the row. Replaces VecComposedPark._file (vec_composed.py:330-345). */
int ebb_composed_file(const EbbComposedState* s, const uint8_t* mask, const double* pos, const double* vel,
                      const float* sf, void* stream);

/* The server layer's pre- and post-tick over the flight park, one thread a world, the park written in place. phase 0:
 * all of 1 and 2 over every slot; 1: the stamps, the queue in order (the duplicate test against the world's last queued
 * call, the rows, CloakBall's bubble, every call but CloakBall applied by the park's own command or setter), then the
 * bubble update; 2: the history over slots [j0, j1) (routes, CloakBall applied, the uncloaks' recipients), so that the
 * host can read the park between segments; 3: the send flags (after the park's tick); 4: a bubble without an
 * interactive ball recorded as dead (before the park's tick); 5: phase 0 then phase 4 (a tick whose park tick
 * follows the pre-tick directly); 6: the queue's test alone (each call's queued flag, rows and CloakBall's bubble,
 * nothing applied: what the pending queries read between ticks). Returns -1 for a bad argument (J outside
 * [0, EBB_SERVER_MAX_SLOTS], a bad phase, range or block), else a cudaError_t. Replaces xbpv_pre_tick
 * (exact_ballpark/vec_server_cuda.cu:615), which exact_ballpark.vec_server_cuda.launch calls (vec_server_cuda.py:307),
 * and VecServer.evolve's dead-bubble test (vec_server.py:1021). */
int ebb_server_tick(const EbbServerState* s, const EbbServerQueue* q, int phase, int64_t j0, int64_t j1, void* stream,
                    int block);

/* glibc 2.34's rand() after srand(seed) (random_r, TYPE_3), one generator a world: a world's state is EBB_RAND_WORDS
 * int32 (the 31-word table, then the front and rear indices). ebb_glibc_srand seeds worlds[W] states from seeds[W]
 * (srandom_r, its 310 discarded draws included); ebb_glibc_rand draws `draws` values a world into out[W][draws],
 * advancing the states. destiny's floatrand (Ball.cpp:19) is rand() / 2147483647.0. Replaces GlibcRandom and
 * glibc_srand (exact_ballpark/glibc_rand.py:14, vec_space.py:148) and vec_space.cu's glibc_rand. */
#define EBB_RAND_WORDS 33
int ebb_glibc_srand(const int64_t* seeds, int64_t worlds, int32_t* state, void* stream);
int ebb_glibc_rand(int32_t* state, int64_t worlds, int64_t draws, int32_t* out, void* stream);

/* SnapOrientation of the rows in mask[n] (nonzero bytes): the rotation turned to the velocity and rolled upright,
 * the old rotation the same, the angular velocities zeroed (at a speed of 1e-6 m/s or less nothing changes). With
 * `fresh`, first the state of a new ball: rotation identity, old rotation rot x RotationQuaternion(angVel,
 * -dt |angVel|), angular velocities kept. Replaces VecOrientPark._snap_orientation and the load's mOldRot
 * (exact_ballpark/vec_orient.py:556, vec_modes.py:256-264). */
int ebb_flight_snap(const EbbFlightState* s, const uint8_t* mask, int fresh, void* stream, int block);

/* SetBallTimeFactor for the rows in mask[n]: time_factor = 0 if mass x agility <= 0, else exp(neg_kdt / (mass x
 * agility)) with glibc's exp, neg_kdt = -friction x dt. Replaces VecOrientPark._decay (vec_orient.py:376). */
int ebb_flight_decay(const EbbFlightState* s, const uint8_t* mask, double neg_kdt, void* stream, int block);

/* glibc 2.34 aarch64's function `func` elementwise on the device, for the tests: 0 sin, 1 cos, 2 log, 3 exp,
 * 4 sincos's sine, 5 sincos's cosine, 6 pow(x, y); 10 expf, 11 logf, 12 sinf, 13 cosf, 14 acosf, 15 atanf,
 * 16 atan2f(y, x), 17 powf(x, y) (floats held in doubles; powf is glibc_powf.cuh:65's g_powf, the combat
 * kernel's mushroom growth). Replaces xbpm_dlibm and xbpo_libm (vec_modes_cuda.cu:779, vec_orient_cuda.cu:520). */
int ebb_libm(int func, int64_t n, const double* x, const double* y, double* out, void* stream, int block);

/* The tape's operations on every world, one thread a world, on `stream` (the park's rows are read and written: the
 * interactive and sensor flags, and a sensor check's radius, put back after it). Replaces xbps_tape_cuda
 * (exact_ballpark/vec_space.py:896). */
int ebb_space_tape(const EbbFlightState* park, const EbbSpaceState* s, const EbbSpaceTape* t, void* stream, int block);

/* One query a world (EbbSpaceQuery), one thread a world, on `stream`; nothing but the answer written. Replaces
 * xbps_query_cuda (exact_ballpark/vec_space.py:938). */
int ebb_space_query(const EbbFlightState* park, const EbbSpaceState* s, const EbbSpaceQuery* q, void* stream,
                    int block);

/* A kernel's resources as loaded on the current device: which 0 the plain tick, 1 the prepass, 2 the tiled tick,
 * 3 the listed-worlds tick, 4 the row move, 7 the combat tick, 8 the composed tick.
 * Replaces xbpm_info (vec_modes_cuda.cu:766). */
int ebb_kernel_info(int which, int* regs, int* local_bytes, int* binary_version, int* ptx_version, int* max_threads);

#ifdef __cplusplus
}
#endif

#endif /* EBB_H */
