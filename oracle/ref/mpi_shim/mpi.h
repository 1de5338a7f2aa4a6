/*
 * Single-rank loopback stand-in for <mpi.h>.
 *
 * Test infrastructure only: it lets the reference's own walk engine and
 * trainer sources compile and run as one process (np = 1) so that the oracle
 * can be checked against them.  Every point-to-point message is sent to rank 0
 * itself: MPI_Isend / MPI_Send enqueue a copy, MPI_Probe / MPI_Recv /
 * MPI_Irecv dequeue it in FIFO order per tag.  Collectives over one rank are
 * copies.  The reference needs loopback delivery even at np = 1 because its
 * walkers are handed to their own partition through the message runtime
 * (graph.hpp distributed_execute) and its footprints through path.hpp
 * assemble_path.
 */
#ifndef FELOG_MPI_SHIM_H
#define FELOG_MPI_SHIM_H

#include <stddef.h>
#include <string.h>
#include <stdio.h>

#ifdef __cplusplus
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <vector>
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct {
  int MPI_SOURCE;
  int MPI_TAG;
  int MPI_ERROR;
  size_t bytes;
} MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_MAX_PROCESSOR_NAME 64
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_IN_PLACE ((void *)1)

#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_THREAD_SERIALIZED 2
#define MPI_THREAD_MULTIPLE 3

/* Datatypes are encoded as their size in bytes (plus a tag in the high bits
 * so distinct types stay distinct values). */
#define FELOG_MPI_TYPE(tag, size) (((tag) << 8) | (size))
#define MPI_CHAR FELOG_MPI_TYPE(1, 1)
#define MPI_BYTE FELOG_MPI_TYPE(2, 1)
#define MPI_UNSIGNED_CHAR FELOG_MPI_TYPE(3, 1)
#define MPI_INT FELOG_MPI_TYPE(4, 4)
#define MPI_UNSIGNED FELOG_MPI_TYPE(5, 4)
#define MPI_FLOAT FELOG_MPI_TYPE(6, 4)
#define MPI_LONG FELOG_MPI_TYPE(7, 8)
#define MPI_UNSIGNED_LONG FELOG_MPI_TYPE(8, 8)
#define MPI_LONG_LONG FELOG_MPI_TYPE(9, 8)
#define MPI_DOUBLE FELOG_MPI_TYPE(10, 8)

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3

static inline size_t felog_mpi_type_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

#ifdef __cplusplus
namespace felog_mpi_shim {
struct Queue {
  std::mutex mu;
  std::condition_variable cv;
  std::map<int, std::deque<std::vector<char>>> by_tag;
};
inline Queue &queue() {
  static Queue q;
  return q;
}
inline void push(const void *buf, size_t bytes, int tag) {
  Queue &q = queue();
  std::vector<char> msg((const char *)buf, (const char *)buf + bytes);
  {
    std::lock_guard<std::mutex> g(q.mu);
    q.by_tag[tag].push_back(std::move(msg));
  }
  q.cv.notify_all();
}
inline size_t peek(int tag) {
  Queue &q = queue();
  std::unique_lock<std::mutex> lk(q.mu);
  q.cv.wait(lk, [&] { return !q.by_tag[tag].empty(); });
  return q.by_tag[tag].front().size();
}
inline size_t pop(void *buf, size_t cap, int tag) {
  Queue &q = queue();
  std::unique_lock<std::mutex> lk(q.mu);
  q.cv.wait(lk, [&] { return !q.by_tag[tag].empty(); });
  std::vector<char> msg = std::move(q.by_tag[tag].front());
  q.by_tag[tag].pop_front();
  size_t n = msg.size() < cap ? msg.size() : cap;
  if (n) memcpy(buf, msg.data(), n);
  return msg.size();
}
}  // namespace felog_mpi_shim

inline int MPI_Init_thread(int *, char ***, int, int *provided) {
  if (provided) *provided = MPI_THREAD_MULTIPLE;
  return MPI_SUCCESS;
}
inline int MPI_Init(int *, char ***) { return MPI_SUCCESS; }
inline int MPI_Finalize() { return MPI_SUCCESS; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return MPI_SUCCESS; }
inline int MPI_Comm_size(MPI_Comm, int *s) { *s = 1; return MPI_SUCCESS; }
inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm *out) { *out = c; return MPI_SUCCESS; }
inline int MPI_Get_processor_name(char *name, int *len) {
  strcpy(name, "loopback");
  *len = 8;
  return MPI_SUCCESS;
}
inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
inline int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (send != MPI_IN_PLACE && send != recv) memmove(recv, send, (size_t)count * felog_mpi_type_size(t));
  return MPI_SUCCESS;
}
inline int MPI_Send(const void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm) {
  felog_mpi_shim::push(buf, (size_t)count * felog_mpi_type_size(t), tag);
  return MPI_SUCCESS;
}
inline int MPI_Isend(const void *buf, int count, MPI_Datatype t, int dst, int tag, MPI_Comm c, MPI_Request *req) {
  if (req) *req = 0;
  return MPI_Send(buf, count, t, dst, tag, c);
}
inline int MPI_Probe(int src, int tag, MPI_Comm, MPI_Status *st) {
  size_t n = felog_mpi_shim::peek(tag);
  if (st) {
    st->MPI_SOURCE = src;
    st->MPI_TAG = tag;
    st->MPI_ERROR = 0;
    st->bytes = n;
  }
  return MPI_SUCCESS;
}
inline int MPI_Get_count(const MPI_Status *st, MPI_Datatype t, int *count) {
  *count = (int)(st->bytes / felog_mpi_type_size(t));
  return MPI_SUCCESS;
}
inline int MPI_Recv(void *buf, int count, MPI_Datatype t, int, int tag, MPI_Comm, MPI_Status *st) {
  size_t n = felog_mpi_shim::pop(buf, (size_t)count * felog_mpi_type_size(t), tag);
  if (st) {
    st->MPI_TAG = tag;
    st->bytes = n;
  }
  return MPI_SUCCESS;
}
inline int MPI_Irecv(void *buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Request *req) {
  if (req) *req = 0;
  return MPI_Recv(buf, count, t, src, tag, c, MPI_STATUS_IGNORE);
}
inline int MPI_Wait(MPI_Request *, MPI_Status *) { return MPI_SUCCESS; }
#endif /* __cplusplus */

#endif
