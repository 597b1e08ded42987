// slab_parts.cuh -- particles of a y-slab held by their owner slab: the
// messages between neighbour slabs and the slab's device state (capi.cu,
// particle_kernels.cu).
#pragma once

#include <vector>

#include "lbrb_internal.cuh"

namespace lbrb {

// ------------------------------------------------- owner-slab particles
// A y-slab holds the particles whose cell lies in its rows.  After each step
// it sends its neighbours two kinds of message, each a SlabMsg header and a
// body:
//   moment rows (SlabMsg::kind MSG_MOM_UP / MSG_MOM_DOWN): planes of nx
//     values from byte MOM_PLANES_OFF on, each MOM plane stride apart.  Up
//     (to the slab above): u, v, T of the top row.  Down (to the slab below):
//     u, v, u^{n-1}, v^{n-1}, T of row 0, then u, v, T of row 1.  A slab's
//     particle stencils reach one row below its rows and two above
//     (periodic in y, as the reference's halos are).
//   hand-off lists (MSG_HAND_UP / MSG_HAND_DOWN): `count` HandoffRec records
//     from byte HAND_RECS_OFF on, the particles that left the slab's rows.
// The receiver checks the header's step and the sender's rows.
struct SlabMsg {
  int count;   // hand-off: records in the list; moments: planes
  int step;    // the sender's step
  int j0, j1;  // the sender's rows [j0, j1) of the domain
  int kind;
  int pad[3];
};
static_assert(sizeof(SlabMsg) == 32, "SlabMsg");
struct HandoffRec {
  double P[9];  // x y u v xo yo uo vo invtau
  int id, type;
};
static_assert(sizeof(HandoffRec) == 80, "HandoffRec");
enum : int { MSG_MOM_UP = 1, MSG_MOM_DOWN = 2, MSG_HAND_UP = 3, MSG_HAND_DOWN = 4 };
constexpr size_t MOM_PLANES_OFF = 256;
constexpr size_t HAND_RECS_OFF = 32;
constexpr int MOM_UP_PLANES = 3, MOM_DOWN_PLANES = 8;
// field tables of the particle kernels: 14 tables of ny_total row pointers,
// u and v for the 3 moment slots (as u^n), u and v again (as u^{n-1}: their
// ghost rows differ), T for the 2 buffers
constexpr int OWN_TABLES = 14;

struct SlabParts {
  int cap = 0;   // particles the slab can hold (a multiple of 128; 0: moment messages only)
  int xcap = 0;  // records per hand-off list
  double* P[2] = {nullptr, nullptr};  // [9][cap]: x y u v xo yo uo vo invtau
  int* id[2] = {nullptr, nullptr};
  int* type[2] = {nullptr, nullptr};
  int pc = 0;               // the current buffer (the step compacts into the other)
  int* cnt = nullptr;       // device: [0] particles kept by the last step, [1] with the received ones
  unsigned char* cls = nullptr;  // [cap]: 0 kept, 1 up, 2 down, 3 none
  int* bcnt = nullptr;      // [cap / 128][3] block counts, then offsets
  unsigned* done = nullptr; // blocks of the particle step finished (reset by its last block)
  void* mom[4] = {nullptr, nullptr, nullptr, nullptr};   // up, down (sent), lo, hi (received)
  void* hand[4] = {nullptr, nullptr, nullptr, nullptr};  // up, down (sent), lo, hi (received)
  size_t mom_pstride = 0, mom_up_bytes = 0, mom_down_bytes = 0, hand_bytes = 0;
  // where the moment rows and hand-off lists are written (up, down): the
  // slab's own send buffers, or, inside lbrb_slab_step, the neighbours'
  // receive buffers directly (null: own)
  void* dst_mom[2] = {nullptr, nullptr};
  void* dst_hand[2] = {nullptr, nullptr};
  void* rows = nullptr;     // device: OWN_TABLES x ny_total row pointers
  void* zrow = nullptr;     // a row of zeros (rows outside the slab's reach)
  // records: per slot nrec_fields x cap doubles, cap ids and the count
  double* d_rec = nullptr;
  int* d_rid = nullptr;
  int* d_rcnt = nullptr;
  double* h_rec = nullptr;
  int* h_rid = nullptr;
  int* h_rcnt = nullptr;
  std::vector<int> rstep;
  std::vector<cudaEvent_t> rev;
  long rhead = 0, rtail = 0;
  // protocol: the step of the last moment pack, particle step, receive and
  // bilinear nudging (lbrb_slab_nudge)
  int mom_step = -1, part_step = 0, recv_step = 0, nudge_step = 0;
  // lbrb_step(h, 2) left the handle at the first of its two steps: the
  // first lbrb_slab_particles_recv moves it on to the second
  bool pair_pending = false;
  cudaEvent_t ev_mom = nullptr, ev_part = nullptr, ev_hand = nullptr;
};

}  // namespace lbrb
