// Single-rank stand-in for the MPI calls the imexlb proxy apps make
// (tgv/src/mpi_view_transfer.cpp, lid_driven_cavity/src/mpi_view_transfer.cpp,
// sphere/src/mpi_view_transfer.cpp, */src/lbm.cpp MPIoutput, */src/lbm.hpp).
// Test infrastructure: it lets the reference's own sources run on one CPU
// process so they can pin this project's restatement.
//
// Semantics at one rank (MPI-3.1 standard):
//   * every rank argument names rank 0; point-to-point messages to self match
//     by tag, the payload is copied when the pair is complete, and
//     MPI_Waitall aborts if any posted message is still unmatched;
//   * a blocking receive with no matching send would deadlock: abort instead;
//   * collectives (Allgather, Reduce) copy the one contribution;
//   * MPI-IO: MPI_File_write writes at the individual file pointer; after
//     MPI_File_set_view the data of MPI_File_write_all lands at the view's
//     displacement.  At one rank the subarray file type covers the whole
//     global array, so the view is contiguous; anything else aborts.
#pragma once

#include <fcntl.h>
#include <time.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef long long MPI_Offset;
typedef int MPIO_Request;
typedef struct {
  int MPI_SOURCE, MPI_TAG, MPI_ERROR;
} MPI_Status;
struct refshim_mpi_file {
  int fd;
  MPI_Offset ptr;
  MPI_Offset disp;
  int etype_size;
};
typedef refshim_mpi_file* MPI_File;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_CHAR 1
#define MPI_INT 2
#define MPI_REAL 3
#define MPI_DOUBLE 4
#define MPI_BYTE 5
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_INFO_NULL 0
#define MPI_MODE_CREATE 1
#define MPI_MODE_WRONLY 4
#define MPI_SEEK_SET 600
#define MPI_ORDER_FORTRAN 57
#define MPI_ORDER_C 56
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)

namespace refshim_mpi {

[[noreturn]] inline void fail(const char* what) {
  std::fprintf(stderr, "refshim mpi: %s\n", what);
  std::abort();
}

struct TypeInfo {
  int size;        // bytes of one element of this type
  bool contiguous; // whole-array subarray or contiguous of contiguous
};

inline std::vector<TypeInfo>& types() {
  static std::vector<TypeInfo> t = {
      {0, true}, {1, true}, {4, true}, {4, true}, {8, true}, {1, true}};
  return t;
}
inline int type_size(MPI_Datatype t) {
  if (t <= 0 || t >= static_cast<int>(types().size())) fail("unknown datatype");
  return types()[t].size;
}

struct Msg {
  const void* sbuf;        // Isend buffer (copied at match time) or null
  std::vector<char> eager; // blocking-send copy
  void* rbuf;
  size_t bytes;
  int tag;
  bool is_send;
  bool done;
};
inline std::vector<Msg>& pending() {
  static std::vector<Msg> p;
  return p;
}
// Try to pair message `m` with a waiting partner of opposite kind and same tag.
inline bool match(Msg& m, int* req_self) {
  auto& p = pending();
  for (size_t k = 0; k < p.size(); ++k) {
    Msg& o = p[k];
    if (o.done || o.is_send == m.is_send || o.tag != m.tag) continue;
    Msg& s = m.is_send ? m : o;
    Msg& r = m.is_send ? o : m;
    if (s.bytes != r.bytes) fail("self message size mismatch");
    const void* src = s.sbuf ? s.sbuf : s.eager.data();
    std::memcpy(r.rbuf, src, r.bytes);
    o.done = true;
    (void)req_self;
    return true;
  }
  return false;
}

}  // namespace refshim_mpi

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_size(MPI_Comm, int* n) {
  *n = 1;
  return 0;
}
inline int MPI_Comm_rank(MPI_Comm, int* r) {
  *r = 0;
  return 0;
}
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline double MPI_Wtime() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
inline int MPI_Allgather(const void* s, int sc, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
  std::memcpy(r, s, static_cast<size_t>(sc) * refshim_mpi::type_size(st));
  return 0;
}
inline int MPI_Reduce(const void* s, void* r, int c, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  std::memcpy(r, s, static_cast<size_t>(c) * refshim_mpi::type_size(t));
  return 0;
}

// Point-to-point to self.  Each posted operation records whether it has been
// matched; MPI_Wait(all) aborts on an unmatched request (a real deadlock).
inline int MPI_Isend(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm,
                     MPI_Request* req) {
  if (dest != 0) refshim_mpi::fail("Isend to a rank other than self");
  refshim_mpi::Msg m{buf, {}, nullptr, static_cast<size_t>(count) * refshim_mpi::type_size(t), tag, true, false};
  m.done = refshim_mpi::match(m, nullptr);
  refshim_mpi::pending().push_back(m);
  *req = 0;
  return 0;
}
inline int MPI_Irecv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Request* req) {
  if (src != 0) refshim_mpi::fail("Irecv from a rank other than self");
  refshim_mpi::Msg m{nullptr, {}, buf, static_cast<size_t>(count) * refshim_mpi::type_size(t), tag, false, false};
  m.done = refshim_mpi::match(m, nullptr);
  refshim_mpi::pending().push_back(m);
  *req = 0;
  return 0;
}
inline int MPI_Send(const void* buf, int count, MPI_Datatype t, int dest, int tag, MPI_Comm) {
  if (dest != 0) refshim_mpi::fail("Send to a rank other than self");
  const size_t bytes = static_cast<size_t>(count) * refshim_mpi::type_size(t);
  refshim_mpi::Msg m{nullptr, std::vector<char>(static_cast<const char*>(buf), static_cast<const char*>(buf) + bytes),
                     nullptr, bytes, tag, true, false};
  m.done = refshim_mpi::match(m, nullptr);
  refshim_mpi::pending().push_back(std::move(m));
  return 0;
}
inline int MPI_Recv(void* buf, int count, MPI_Datatype t, int src, int tag, MPI_Comm, MPI_Status*) {
  if (src != 0) refshim_mpi::fail("Recv from a rank other than self");
  refshim_mpi::Msg m{nullptr, {}, buf, static_cast<size_t>(count) * refshim_mpi::type_size(t), tag, false, false};
  if (!refshim_mpi::match(m, nullptr)) refshim_mpi::fail("blocking Recv with no matching send (deadlock)");
  return 0;
}
inline int MPI_Wait(MPI_Request*, MPI_Status*) {
  // Completion is checked collectively; an Isend to self is complete once posted.
  return 0;
}
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) {
  // At one rank every send and receive must have found its partner by now.
  auto& p = refshim_mpi::pending();
  for (auto& m : p)
    if (!m.done) refshim_mpi::fail("Waitall with unmatched self messages (deadlock)");
  p.clear();
  return 0;
}

// Derived datatypes: only the shapes MPIoutput builds are accepted.
inline int MPI_Type_create_subarray(int ndims, const int* sizes, const int* subsizes, const int* starts, int,
                                    MPI_Datatype old, MPI_Datatype* out) {
  long n = 1;
  for (int d = 0; d < ndims; ++d) {
    if (starts[d] != 0 || subsizes[d] != sizes[d]) refshim_mpi::fail("subarray is not the whole array");
    n *= sizes[d];
  }
  refshim_mpi::types().push_back({static_cast<int>(n * refshim_mpi::type_size(old)), true});
  *out = static_cast<int>(refshim_mpi::types().size()) - 1;
  return 0;
}
inline int MPI_Type_contiguous(int count, MPI_Datatype old, MPI_Datatype* out) {
  refshim_mpi::types().push_back({count * refshim_mpi::type_size(old), true});
  *out = static_cast<int>(refshim_mpi::types().size()) - 1;
  return 0;
}
inline int MPI_Type_commit(MPI_Datatype*) { return 0; }
inline int MPI_Type_free(MPI_Datatype*) { return 0; }

inline int MPI_File_open(MPI_Comm, const char* name, int amode, MPI_Info, MPI_File* fh) {
  int flags = O_WRONLY;
  if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
  int fd = ::open(name, flags, 0644);
  if (fd < 0) refshim_mpi::fail("MPI_File_open failed");
  *fh = new refshim_mpi_file{fd, 0, 0, 1};
  return 0;
}
inline int MPI_File_seek(MPI_File fh, MPI_Offset off, int) {
  fh->ptr = off;
  return 0;
}
inline int MPI_File_write(MPI_File fh, const void* buf, int count, MPI_Datatype t, MPI_Status*) {
  const size_t bytes = static_cast<size_t>(count) * refshim_mpi::type_size(t);
  const MPI_Offset at = fh->disp + fh->ptr * fh->etype_size;
  if (::pwrite(fh->fd, buf, bytes, at) != static_cast<ssize_t>(bytes)) refshim_mpi::fail("pwrite");
  fh->ptr += static_cast<MPI_Offset>(bytes / fh->etype_size);
  return 0;
}
inline int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype, const char*,
                             MPI_Info) {
  if (!refshim_mpi::types()[filetype].contiguous) refshim_mpi::fail("non-contiguous file view");
  fh->disp = disp;
  fh->etype_size = refshim_mpi::type_size(etype);
  fh->ptr = 0;
  return 0;
}
inline int MPI_File_write_all(MPI_File fh, const void* buf, int count, MPI_Datatype t, MPI_Status* s) {
  return MPI_File_write(fh, buf, count, t, s);
}
inline int MPI_File_close(MPI_File* fh) {
  ::close((*fh)->fd);
  delete *fh;
  *fh = nullptr;
  return 0;
}
