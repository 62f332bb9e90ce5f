// Size-1 implementation of the MPI names declared in mpi.h (TEST
// INFRASTRUCTURE ONLY: it lets the reference's own sources link as the CPU
// oracle).  Every communicator has one process, rank 0.  Collectives copy the
// send buffer to the receive buffer (nothing when the buffers coincide or the
// send buffer is MPI_IN_PLACE); a reduction over one process is its operand,
// so created operators are recorded but never applied.  Point-to-point
// messages can only go to self: a send is buffered at once and a receive
// takes the oldest buffered message with a matching tag.
#include "mpi.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

namespace {

bool g_init = false, g_final = false;

size_t type_size(MPI_Datatype t) {
  switch (t) {
    case MPI_BYTE: case MPI_CHAR: case MPI_UNSIGNED_CHAR: return 1;
    case MPI_INT: case MPI_UNSIGNED: return 4;
    case MPI_LONG: case MPI_UNSIGNED_LONG: case MPI_LONG_LONG_INT: case MPI_UNSIGNED_LONG_LONG: return 8;
    case MPI_FLOAT: return 4;
    case MPI_DOUBLE: return 8;
    case MPI_COMPLEX: return 8;
    case MPI_DOUBLE_COMPLEX: return 16;
    case MPI_FLOAT_INT: return 8;
    case MPI_DOUBLE_INT: return 16;
    case MPI_2INT: return 8;
    default:
      std::fprintf(stderr, "single-process MPI: unknown datatype %d\n", t);
      std::abort();
  }
}

void copy(const void* src, void* dst, int count, MPI_Datatype t) {
  if (src == MPI_IN_PLACE || src == dst || count <= 0) return;
  std::memmove(dst, src, (size_t)count * type_size(t));
}

struct Message {
  int tag;
  std::vector<char> data;
};
std::deque<Message> g_mailbox;  // messages sent to self, oldest first

struct PendingRecv {
  void* buf;
  size_t cap;
  int tag;
  bool done;
  int bytes;
  int src_tag;
};
std::map<int, PendingRecv> g_requests;  // request id -> pending receive (sends complete at once)
int g_next_request = 1;
int g_next_op = 100;

bool take(int tag, void* buf, size_t cap, int* bytes, int* got_tag) {
  for (auto it = g_mailbox.begin(); it != g_mailbox.end(); ++it) {
    if (tag != MPI_ANY_TAG && it->tag != tag) continue;
    const size_t n = it->data.size() < cap ? it->data.size() : cap;
    if (n) std::memcpy(buf, it->data.data(), n);
    *bytes = (int)n;
    *got_tag = it->tag;
    g_mailbox.erase(it);
    return true;
  }
  return false;
}

void post(const void* buf, int count, MPI_Datatype t, int tag) {
  Message m;
  m.tag = tag;
  m.data.resize((size_t)count * type_size(t));
  if (!m.data.empty()) std::memcpy(m.data.data(), buf, m.data.size());
  g_mailbox.push_back(std::move(m));
  // complete receives that were posted before this message
  for (auto& kv : g_requests) {
    PendingRecv& r = kv.second;
    if (!r.done && take(r.tag, r.buf, r.cap, &r.bytes, &r.src_tag)) r.done = true;
  }
}

void set_status(MPI_Status* st, int tag, int bytes) {
  if (st == MPI_STATUS_IGNORE) return;
  st->MPI_SOURCE = 0;
  st->MPI_TAG = tag;
  st->MPI_ERROR = MPI_SUCCESS;
  st->count_bytes = bytes;
}

int fail(const char* what) {
  std::fprintf(stderr, "single-process MPI: %s\n", what);
  std::abort();
}

}  // namespace

extern "C" {

int MPI_Init(int*, char***) { g_init = true; return MPI_SUCCESS; }
int MPI_Init_thread(int*, char***, int required, int* provided) {
  g_init = true;
  if (provided) *provided = required;
  return MPI_SUCCESS;
}
int MPI_Initialized(int* flag) { *flag = g_init ? 1 : 0; return MPI_SUCCESS; }
int MPI_Finalized(int* flag) { *flag = g_final ? 1 : 0; return MPI_SUCCESS; }
int MPI_Finalize(void) { g_final = true; return MPI_SUCCESS; }
int MPI_Query_thread(int* provided) { *provided = MPI_THREAD_MULTIPLE; return MPI_SUCCESS; }
double MPI_Wtime(void) {
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}
int MPI_Error_string(int code, char* s, int* len) {
  *len = std::snprintf(s, MPI_MAX_ERROR_STRING, "single-process MPI error %d", code);
  return MPI_SUCCESS;
}
int MPI_Errhandler_set(MPI_Comm, MPI_Errhandler) { return MPI_SUCCESS; }
int MPI_Comm_set_errhandler(MPI_Comm, MPI_Errhandler) { return MPI_SUCCESS; }

int MPI_Comm_size(MPI_Comm, int* size) { *size = 1; return MPI_SUCCESS; }
int MPI_Comm_rank(MPI_Comm, int* rank) { *rank = 0; return MPI_SUCCESS; }
int MPI_Comm_dup(MPI_Comm comm, MPI_Comm* out) { *out = comm; return MPI_SUCCESS; }
int MPI_Comm_split(MPI_Comm comm, int color, int, MPI_Comm* out) {
  *out = color == MPI_UNDEFINED ? MPI_COMM_NULL : comm;
  return MPI_SUCCESS;
}
int MPI_Comm_create(MPI_Comm comm, MPI_Group group, MPI_Comm* out) {
  *out = group == MPI_GROUP_EMPTY ? MPI_COMM_NULL : comm;
  return MPI_SUCCESS;
}
int MPI_Comm_free(MPI_Comm* comm) { *comm = MPI_COMM_NULL; return MPI_SUCCESS; }
int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* result) {
  *result = a == b ? MPI_IDENT : MPI_CONGRUENT;
  return MPI_SUCCESS;
}
int MPI_Comm_group(MPI_Comm, MPI_Group* group) { *group = 2; return MPI_SUCCESS; }
int MPI_Cart_create(MPI_Comm comm, int, const int*, const int*, int, MPI_Comm* cart) { *cart = comm; return MPI_SUCCESS; }
int MPI_Cart_sub(MPI_Comm comm, const int*, MPI_Comm* out) { *out = comm; return MPI_SUCCESS; }

// groups: MPI_GROUP_EMPTY (size 0) or a group holding the one process
int MPI_Group_size(MPI_Group g, int* size) { *size = g == MPI_GROUP_EMPTY ? 0 : 1; return MPI_SUCCESS; }
int MPI_Group_rank(MPI_Group g, int* rank) { *rank = g == MPI_GROUP_EMPTY ? MPI_UNDEFINED : 0; return MPI_SUCCESS; }
int MPI_Group_incl(MPI_Group, int n, const int*, MPI_Group* out) {
  *out = n > 0 ? 2 : MPI_GROUP_EMPTY;
  return MPI_SUCCESS;
}
int MPI_Group_difference(MPI_Group a, MPI_Group b, MPI_Group* out) {
  *out = (a == MPI_GROUP_EMPTY || b != MPI_GROUP_EMPTY) ? MPI_GROUP_EMPTY : a;
  return MPI_SUCCESS;
}
int MPI_Group_translate_ranks(MPI_Group, int n, const int* ra, MPI_Group b, int* rb) {
  for (int i = 0; i < n; ++i) rb[i] = (b == MPI_GROUP_EMPTY || ra[i] != 0) ? MPI_UNDEFINED : 0;
  return MPI_SUCCESS;
}
int MPI_Group_free(MPI_Group* g) { *g = MPI_GROUP_NULL; return MPI_SUCCESS; }

int MPI_Op_create(MPI_User_function*, int, MPI_Op* op) { *op = g_next_op++; return MPI_SUCCESS; }
int MPI_Op_free(MPI_Op* op) { *op = MPI_OP_NULL; return MPI_SUCCESS; }

int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm) {
  if (dest != 0) return fail("send to a rank other than 0");
  post(buf, count, t, tag);
  return MPI_SUCCESS;
}
int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request* req) {
  *req = MPI_REQUEST_NULL;
  return MPI_Send(buf, count, t, dest, tag, c);
}
int MPI_Issend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm c, MPI_Request* req) {
  return MPI_Isend(buf, count, t, dest, tag, c, req);
}
int MPI_Recv(void* buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm, MPI_Status* st) {
  if (source != 0 && source != MPI_ANY_SOURCE) return fail("receive from a rank other than 0");
  int bytes = 0, got = 0;
  if (!take(tag, buf, (size_t)count * type_size(t), &bytes, &got)) return fail("receive without a matching send");
  set_status(st, got, bytes);
  return MPI_SUCCESS;
}
int MPI_Irecv(void* buf, int count, MPI_Datatype t, int source, int tag, MPI_Comm, MPI_Request* req) {
  if (source != 0 && source != MPI_ANY_SOURCE) return fail("receive from a rank other than 0");
  PendingRecv r{buf, (size_t)count * type_size(t), tag, false, 0, 0};
  r.done = take(tag, buf, r.cap, &r.bytes, &r.src_tag);
  const int id = g_next_request++;
  g_requests[id] = r;
  *req = id;
  return MPI_SUCCESS;
}
int MPI_Sendrecv(const void* sbuf, int scount, MPI_Datatype stype, int dest, int stag, void* rbuf, int rcount,
                 MPI_Datatype rtype, int source, int rtag, MPI_Comm comm, MPI_Status* st) {
  MPI_Send(sbuf, scount, stype, dest, stag, comm);
  return MPI_Recv(rbuf, rcount, rtype, source, rtag, comm, st);
}
int MPI_Sendrecv_replace(void* buf, int count, MPI_Datatype t, int dest, int stag, int source, int rtag,
                         MPI_Comm comm, MPI_Status* st) {
  MPI_Send(buf, count, t, dest, stag, comm);
  return MPI_Recv(buf, count, t, source, rtag, comm, st);
}
int MPI_Iprobe(int, int tag, MPI_Comm, int* flag, MPI_Status* st) {
  *flag = 0;
  for (const auto& m : g_mailbox)
    if (tag == MPI_ANY_TAG || m.tag == tag) {
      *flag = 1;
      set_status(st, m.tag, (int)m.data.size());
      break;
    }
  return MPI_SUCCESS;
}
int MPI_Get_count(const MPI_Status* st, MPI_Datatype t, int* count) {
  *count = st->count_bytes / (int)type_size(t);
  return MPI_SUCCESS;
}
int MPI_Test(MPI_Request* req, int* flag, MPI_Status* st) {
  if (*req == MPI_REQUEST_NULL) { *flag = 1; set_status(st, 0, 0); return MPI_SUCCESS; }
  auto it = g_requests.find(*req);
  if (it == g_requests.end()) return fail("unknown request");
  *flag = it->second.done ? 1 : 0;
  if (*flag) {
    set_status(st, it->second.src_tag, it->second.bytes);
    g_requests.erase(it);
    *req = MPI_REQUEST_NULL;
  }
  return MPI_SUCCESS;
}
int MPI_Wait(MPI_Request* req, MPI_Status* st) {
  int flag = 0;
  MPI_Test(req, &flag, st);
  if (!flag) return fail("wait on a receive that no send matches");
  return MPI_SUCCESS;
}
int MPI_Waitall(int count, MPI_Request* reqs, MPI_Status* sts) {
  for (int i = 0; i < count; ++i) MPI_Wait(&reqs[i], sts == MPI_STATUSES_IGNORE ? MPI_STATUS_IGNORE : &sts[i]);
  return MPI_SUCCESS;
}

int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
int MPI_Ibcast(void*, int, MPI_Datatype, int, MPI_Comm, MPI_Request* req) { *req = MPI_REQUEST_NULL; return MPI_SUCCESS; }
int MPI_Gather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int, MPI_Datatype, int, MPI_Comm) {
  copy(sbuf, rbuf, scount, stype);
  return MPI_SUCCESS;
}
int MPI_Igather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int rcount, MPI_Datatype rtype,
                int root, MPI_Comm comm, MPI_Request* req) {
  *req = MPI_REQUEST_NULL;
  return MPI_Gather(sbuf, scount, stype, rbuf, rcount, rtype, root, comm);
}
int MPI_Gatherv(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, const int*, const int* displs,
                MPI_Datatype rtype, int, MPI_Comm) {
  if (sbuf != MPI_IN_PLACE) copy(sbuf, static_cast<char*>(rbuf) + (size_t)displs[0] * type_size(rtype), scount, stype);
  return MPI_SUCCESS;
}
int MPI_Allgather(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int, MPI_Datatype, MPI_Comm) {
  copy(sbuf, rbuf, scount, stype);
  return MPI_SUCCESS;
}
int MPI_Allgatherv(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, const int*, const int* displs,
                   MPI_Datatype rtype, MPI_Comm) {
  if (sbuf != MPI_IN_PLACE) copy(sbuf, static_cast<char*>(rbuf) + (size_t)displs[0] * type_size(rtype), scount, stype);
  return MPI_SUCCESS;
}
int MPI_Scatter(const void* sbuf, int, MPI_Datatype, void* rbuf, int rcount, MPI_Datatype rtype, int, MPI_Comm) {
  if (rbuf != MPI_IN_PLACE) copy(sbuf, rbuf, rcount, rtype);
  return MPI_SUCCESS;
}
int MPI_Alltoall(const void* sbuf, int scount, MPI_Datatype stype, void* rbuf, int, MPI_Datatype, MPI_Comm) {
  copy(sbuf, rbuf, scount, stype);
  return MPI_SUCCESS;
}
int MPI_Alltoallv(const void* sbuf, const int* scounts, const int* sdispls, MPI_Datatype stype, void* rbuf,
                  const int*, const int* rdispls, MPI_Datatype rtype, MPI_Comm) {
  if (sbuf == MPI_IN_PLACE) return MPI_SUCCESS;
  copy(static_cast<const char*>(sbuf) + (size_t)sdispls[0] * type_size(stype),
       static_cast<char*>(rbuf) + (size_t)rdispls[0] * type_size(rtype), scounts[0], stype);
  return MPI_SUCCESS;
}
int MPI_Reduce(const void* sbuf, void* rbuf, int count, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  copy(sbuf, rbuf, count, t);
  return MPI_SUCCESS;
}
int MPI_Allreduce(const void* sbuf, void* rbuf, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  copy(sbuf, rbuf, count, t);
  return MPI_SUCCESS;
}
int MPI_Reduce_scatter(const void* sbuf, void* rbuf, const int* rcounts, MPI_Datatype t, MPI_Op, MPI_Comm) {
  copy(sbuf, rbuf, rcounts[0], t);
  return MPI_SUCCESS;
}
int MPI_Reduce_scatter_block(const void* sbuf, void* rbuf, int rcount, MPI_Datatype t, MPI_Op, MPI_Comm) {
  copy(sbuf, rbuf, rcount, t);
  return MPI_SUCCESS;
}

}  // extern "C"
