/*
 * mpi_stub.c -- the MPI routines LAMB calls, for exactly one rank, with the
 * Fortran calling convention of gfortran (lower-case name + '_', every
 * argument by reference, the hidden length of each CHARACTER argument
 * appended as size_t).  Together with mpif.h this lets a single-rank LAMB
 * build link without an MPI library, so that its lamb_multiply can call the
 * B200 library through the ISO_C_BINDING module.
 *
 * Semantics at one rank: the communicator has size 1 and rank 0; Bcast does
 * nothing; Allreduce / Allgather / Alltoall(v) copy the send buffer to the
 * receive buffer; Send / Isend to oneself copy the message into a queue and
 * Irecv + Test match the oldest queued message with a fitting tag; windows
 * are local memory (lock / unlock / fence do nothing); Alloc_mem / Free_mem
 * are malloc / free; MPI-IO opens, reads and closes plain files.
 *
 * Build: gcc -O2 -fPIC -shared mpi_stub.c -o libmpi_stub.so
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int32_t fint;

/* The constant table shared with mpif.h (the test compares the two). */
static const struct { const char* name; int64_t value; } k_consts[] = {
    {"MPI_SUCCESS", 0}, {"MPI_ERR_OTHER", 15}, {"MPI_COMM_WORLD", 91}, {"MPI_COMM_SELF", 92},
    {"MPI_COMM_NULL", 0}, {"MPI_ANY_SOURCE", -1}, {"MPI_ANY_TAG", -1}, {"MPI_UNDEFINED", -32766},
    {"MPI_PROC_NULL", -2}, {"MPI_STATUS_SIZE", 6}, {"MPI_SOURCE", 1}, {"MPI_TAG", 2}, {"MPI_ERROR", 3},
    {"MPI_ADDRESS_KIND", 8}, {"MPI_OFFSET_KIND", 8}, {"MPI_INFO_NULL", 0}, {"MPI_ERRORS_RETURN", 2},
    {"MPI_ERRORS_ARE_FATAL", 1}, {"MPI_MAX_ERROR_STRING", 256}, {"MPI_CHARACTER", 101}, {"MPI_INTEGER", 204},
    {"MPI_REAL", 304}, {"MPI_DOUBLE_PRECISION", 308}, {"MPI_INTEGER1", 201}, {"MPI_INTEGER2", 202},
    {"MPI_INTEGER4", 204}, {"MPI_INTEGER8", 208}, {"MPI_REAL4", 304}, {"MPI_REAL8", 308}, {"MPI_REAL16", 316},
    {"MPI_COMPLEX", 408}, {"MPI_COMPLEX8", 408}, {"MPI_COMPLEX16", 416}, {"MPI_LOGICAL", 504}, {"MPI_BYTE", 601},
    {"MPI_MAX", 1}, {"MPI_MIN", 2}, {"MPI_SUM", 3}, {"MPI_PROD", 4}, {"MPI_LOCK_EXCLUSIVE", 1},
    {"MPI_LOCK_SHARED", 2}, {"MPI_MODE_NOCHECK", 1024}, {"MPI_MODE_NOSTORE", 2048}, {"MPI_MODE_NOPUT", 4096},
    {"MPI_MODE_NOPRECEDE", 8192}, {"MPI_MODE_NOSUCCEED", 16384}, {"MPI_MODE_RDONLY", 2}, {"MPI_MODE_RDWR", 8},
    {"MPI_MODE_WRONLY", 4}, {"MPI_MODE_CREATE", 1},
};

int lamb_mpi_stub_constant(const char* name, int64_t* value) {
  for (size_t i = 0; i < sizeof(k_consts) / sizeof(k_consts[0]); ++i)
    if (strcmp(k_consts[i].name, name) == 0) { *value = k_consts[i].value; return 0; }
  return 1;
}

enum { OK = 0, ERR = 15, COMM_WORLD = 91, COMM_SELF = 92, COMM_NULL = 0, ANY = -1 };

/* Bytes of one element of a datatype code (size + 100 * kind tag); 0 if unknown. */
static int64_t type_bytes(fint t) {
  const int kind = t / 100, sz = t % 100;
  if (kind < 1 || kind > 6 || sz < 1 || sz > 16) return 0;
  return sz;
}

static int valid_comm(fint c) { return c == COMM_WORLD || c == COMM_SELF || c >= 1000; }

/* ---- environment ---------------------------------------------------------- */
static int g_inited = 0, g_finalized = 0;
static fint g_next_comm = 1000;

void mpi_init_(fint* ierr) { g_inited = 1; *ierr = OK; }
void mpi_initialized_(fint* flag, fint* ierr) { *flag = g_inited; *ierr = OK; }
void mpi_finalize_(fint* ierr) { g_finalized = 1; *ierr = OK; }
void mpi_comm_size_(fint* comm, fint* size, fint* ierr) { *size = 1; *ierr = valid_comm(*comm) ? OK : ERR; }
void mpi_comm_rank_(fint* comm, fint* rank, fint* ierr) { *rank = 0; *ierr = valid_comm(*comm) ? OK : ERR; }
void mpi_comm_dup_(fint* comm, fint* newcomm, fint* ierr) {
  *ierr = valid_comm(*comm) ? OK : ERR;
  *newcomm = *ierr == OK ? g_next_comm++ : COMM_NULL;
}
void mpi_comm_free_(fint* comm, fint* ierr) { *ierr = valid_comm(*comm) ? OK : ERR; *comm = COMM_NULL; }
void mpi_errhandler_set_(fint* comm, fint* handler, fint* ierr) { (void)handler; *ierr = valid_comm(*comm) ? OK : ERR; }
void mpi_error_string_(fint* code, char* str, fint* len, fint* ierr, size_t str_len) {
  char buf[128];
  snprintf(buf, sizeof buf, "MPI error %d (single-rank stub)", (int)*code);
  size_t n = strlen(buf);
  if (n > str_len) n = str_len;
  memcpy(str, buf, n);
  if (str_len > n) memset(str + n, ' ', str_len - n);
  *len = (fint)n;
  *ierr = OK;
}
void mpi_type_size_(fint* type, fint* size, fint* ierr) {
  const int64_t b = type_bytes(*type);
  *size = (fint)b;
  *ierr = b ? OK : ERR;
}
void mpi_barrier_(fint* comm, fint* ierr) { *ierr = valid_comm(*comm) ? OK : ERR; }

/* ---- collectives: one rank sends to itself ----------------------------- */
static fint copy_elems(const void* src, void* dst, fint count, fint type) {
  const int64_t b = type_bytes(type);
  if (!b || count < 0) return ERR;
  if (src != dst && count) memmove(dst, src, (size_t)(b * count));
  return OK;
}
void mpi_bcast_(void* buf, fint* count, fint* type, fint* root, fint* comm, fint* ierr) {
  (void)buf;
  *ierr = (*root == 0 && valid_comm(*comm) && type_bytes(*type) && *count >= 0) ? OK : ERR;
}
void mpi_allreduce_(void* sbuf, void* rbuf, fint* count, fint* type, fint* op, fint* comm, fint* ierr) {
  *ierr = (*op >= 1 && *op <= 4 && valid_comm(*comm)) ? copy_elems(sbuf, rbuf, *count, *type) : ERR;
}
void mpi_allgather_(void* sbuf, fint* scount, fint* stype, void* rbuf, fint* rcount, fint* rtype, fint* comm,
                    fint* ierr) {
  (void)rcount; (void)rtype;
  *ierr = valid_comm(*comm) ? copy_elems(sbuf, rbuf, *scount, *stype) : ERR;
}
void mpi_alltoall_(void* sbuf, fint* scount, fint* stype, void* rbuf, fint* rcount, fint* rtype, fint* comm,
                   fint* ierr) {
  mpi_allgather_(sbuf, scount, stype, rbuf, rcount, rtype, comm, ierr);
}
void mpi_alltoallv_(char* sbuf, fint* scounts, fint* sdispls, fint* stype, char* rbuf, fint* rcounts, fint* rdispls,
                    fint* rtype, fint* comm, fint* ierr) {
  (void)rcounts;
  const int64_t sb = type_bytes(*stype), rb = type_bytes(*rtype);
  if (!valid_comm(*comm) || !sb || !rb) { *ierr = ERR; return; }
  *ierr = copy_elems(sbuf + sb * sdispls[0], rbuf + rb * rdispls[0], scounts[0], *stype);
}

/* ---- point to point with oneself --------------------------------------------- */
typedef struct msg { fint tag; int64_t bytes; char* data; struct msg* next; } msg;
static msg *g_head = NULL, *g_tail = NULL;
typedef struct { int used, is_recv; void* buf; int64_t cap; fint tag; } req;
#define MAX_REQ 4096
static req g_req[MAX_REQ];

static fint enqueue(const void* buf, fint count, fint type, fint dest, fint tag) {
  const int64_t b = type_bytes(type);
  if (!b || count < 0 || (dest != 0 && dest != -2)) return ERR;
  if (dest == -2) return OK;  /* MPI_PROC_NULL */
  msg* m = (msg*)malloc(sizeof(msg));
  m->tag = tag;
  m->bytes = b * count;
  m->data = (char*)malloc((size_t)(m->bytes ? m->bytes : 1));
  if (m->bytes) memcpy(m->data, buf, (size_t)m->bytes);
  m->next = NULL;
  if (g_tail) g_tail->next = m; else g_head = m;
  g_tail = m;
  return OK;
}
static fint new_req(int is_recv, void* buf, int64_t cap, fint tag) {
  for (fint i = 1; i < MAX_REQ; ++i)
    if (!g_req[i].used) {
      g_req[i] = (req){1, is_recv, buf, cap, tag};
      return i;
    }
  return 0;
}
void mpi_send_(void* buf, fint* count, fint* type, fint* dest, fint* tag, fint* comm, fint* ierr) {
  *ierr = valid_comm(*comm) ? enqueue(buf, *count, *type, *dest, *tag) : ERR;
}
void mpi_isend_(void* buf, fint* count, fint* type, fint* dest, fint* tag, fint* comm, fint* request, fint* ierr) {
  *ierr = valid_comm(*comm) ? enqueue(buf, *count, *type, *dest, *tag) : ERR;
  *request = *ierr == OK ? new_req(0, NULL, 0, *tag) : 0;
  if (*ierr == OK && !*request) *ierr = ERR;
}
void mpi_irecv_(void* buf, fint* count, fint* type, fint* source, fint* tag, fint* comm, fint* request, fint* ierr) {
  const int64_t b = type_bytes(*type);
  if (!valid_comm(*comm) || !b || *count < 0 || (*source != 0 && *source != ANY)) { *ierr = ERR; *request = 0; return; }
  *request = new_req(1, buf, b * *count, *tag);
  *ierr = *request ? OK : ERR;
}
void mpi_test_(fint* request, fint* flag, fint* status, fint* ierr) {
  *ierr = OK;
  const fint r = *request;
  if (r <= 0 || r >= MAX_REQ || !g_req[r].used) { *flag = 1; return; }  /* null request: complete */
  req* q = &g_req[r];
  if (!q->is_recv) {
    q->used = 0;
    *request = 0;
    *flag = 1;
    return;
  }
  msg *prev = NULL, *m = g_head;
  while (m && !(q->tag == ANY || m->tag == q->tag)) { prev = m; m = m->next; }
  if (!m) { *flag = 0; return; }
  const int64_t n = m->bytes < q->cap ? m->bytes : q->cap;
  if (n) memcpy(q->buf, m->data, (size_t)n);
  status[0] = 0;                       /* MPI_SOURCE */
  status[1] = m->tag;                  /* MPI_TAG */
  status[2] = m->bytes > q->cap ? ERR : OK;  /* MPI_ERROR (truncation) */
  status[3] = (fint)(n & 0x7fffffff);  /* bytes received, low / high words */
  status[4] = (fint)(n >> 31);
  if (prev) prev->next = m->next; else g_head = m->next;
  if (g_tail == m) g_tail = prev;
  free(m->data);
  free(m);
  q->used = 0;
  *request = 0;
  *flag = 1;
}
void mpi_get_count_(fint* status, fint* type, fint* count, fint* ierr) {
  const int64_t b = type_bytes(*type);
  const int64_t n = (int64_t)status[3] + ((int64_t)status[4] << 31);
  if (!b) { *ierr = ERR; return; }
  *count = n % b ? -32766 : (fint)(n / b);
  *ierr = OK;
}

/* ---- one-sided windows: local memory -------------------------------------- */
static fint g_next_win = 1;
void mpi_win_create_(void* base, int64_t* size, fint* disp_unit, fint* info, fint* comm, fint* win, fint* ierr) {
  (void)base; (void)info;
  *ierr = (valid_comm(*comm) && *size >= 0 && *disp_unit > 0) ? OK : ERR;
  *win = *ierr == OK ? g_next_win++ : 0;
}
void mpi_win_free_(fint* win, fint* ierr) { *ierr = *win > 0 ? OK : ERR; *win = 0; }
void mpi_win_lock_(fint* lock_type, fint* rank, fint* assert_, fint* win, fint* ierr) {
  (void)assert_;
  *ierr = (*win > 0 && *rank == 0 && (*lock_type == 1 || *lock_type == 2)) ? OK : ERR;
}
void mpi_win_unlock_(fint* rank, fint* win, fint* ierr) { *ierr = (*win > 0 && *rank == 0) ? OK : ERR; }
void mpi_win_fence_(fint* assert_, fint* win, fint* ierr) { (void)assert_; *ierr = *win > 0 ? OK : ERR; }
void mpi_alloc_mem_(int64_t* size, fint* info, void** baseptr, fint* ierr) {
  (void)info;
  *baseptr = *size >= 0 ? malloc((size_t)(*size > 0 ? *size : 1)) : NULL;
  *ierr = *baseptr ? OK : ERR;
}
void mpi_free_mem_(void* base, fint* ierr) { free(base); *ierr = OK; }

/* ---- MPI-IO on plain files ------------------------------------------------------ */
#define MAX_FILES 64
static FILE* g_files[MAX_FILES];
void mpi_file_open_(fint* comm, const char* name, fint* amode, fint* info, fint* fh, fint* ierr, size_t name_len) {
  (void)info;
  *fh = 0;
  if (!valid_comm(*comm)) { *ierr = ERR; return; }
  size_t n = name_len;
  while (n > 0 && (name[n - 1] == ' ' || name[n - 1] == '\0')) --n;
  char* path = (char*)malloc(n + 1);
  memcpy(path, name, n);
  path[n] = '\0';
  const char* mode = (*amode & 2) ? "rb" : (*amode & 8) ? "r+b" : "wb";
  FILE* f = fopen(path, mode);
  free(path);
  if (!f) { *ierr = ERR; return; }
  for (fint i = 1; i < MAX_FILES; ++i)
    if (!g_files[i]) { g_files[i] = f; *fh = i; *ierr = OK; return; }
  fclose(f);
  *ierr = ERR;
}
void mpi_file_read_(fint* fh, void* buf, fint* count, fint* type, fint* status, fint* ierr) {
  const int64_t b = type_bytes(*type);
  if (*fh <= 0 || *fh >= MAX_FILES || !g_files[*fh] || !b || *count < 0) { *ierr = ERR; return; }
  const size_t got = fread(buf, 1, (size_t)(b * *count), g_files[*fh]);
  status[0] = 0;
  status[1] = ANY;
  status[2] = OK;
  status[3] = (fint)(got & 0x7fffffff);
  status[4] = (fint)((int64_t)got >> 31);
  *ierr = OK;
}
void mpi_file_close_(fint* fh, fint* ierr) {
  if (*fh <= 0 || *fh >= MAX_FILES || !g_files[*fh]) { *ierr = ERR; return; }
  fclose(g_files[*fh]);
  g_files[*fh] = NULL;
  *fh = 0;
  *ierr = OK;
}
