/*
 * ns2d_h5.c -- HDF5 file writer for the solver's output (include/ns2d_h5.h).
 *
 * Written from the published HDF5 file-format specification (format version
 * 0 structures):
 *   - superblock version 0, 8-byte offsets and lengths, group leaf node K = 4,
 *     group internal node K = 16;
 *   - version-1 object headers (16-byte prefix, messages 8-byte aligned);
 *   - groups as symbol tables: a local heap ("HEAP") holding the link names,
 *     symbol-table nodes ("SNOD", up to 2 * leaf K entries, sorted by name)
 *     indexed by a version-1 B-tree of type 0 ("TREE", up to 2 * internal K
 *     children per node, keys = heap offsets of names);
 *   - datasets: dataspace (v1), datatype (v1: IEEE double, 32-bit int, or the
 *     {r, i} compound of Solver/src/hdf5_funcs.c:1837-1868), fill value (v2,
 *     undefined), layout (v3, contiguous) and attribute (v1) messages.
 * Raw data goes to the end of the file as it is written; metadata is written
 * after it on flush, children before parents, and the superblock last.
 */
#include "ns2d_h5.h"

#include <errno.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define H5_UNDEF 0xffffffffffffffffull
#define LEAF_K 4
#define NODE_K 16
#define SNOD_CAP (2 * LEAF_K)
#define BT_CAP (2 * NODE_K)
#define ENTRY_SIZE 40
#define SNOD_SIZE (8 + SNOD_CAP * ENTRY_SIZE)
#define BT_SIZE (24 + (BT_CAP + 1) * 8 + BT_CAP * 8)
#define SB_SIZE 96

typedef struct h5_attr {
    char* name;
    double value;
} h5_attr;

typedef struct h5_obj {
    int is_group;
    char* name;
    struct h5_obj** kids;
    int nkids, capkids;
    h5_attr* attrs;
    int nattrs, capattrs;
    /* dataset */
    int type, rank;
    uint64_t dims[8];
    uint64_t data_addr, data_size;
    /* set on flush */
    uint64_t oh_addr, btree_addr, heap_addr;
} h5_obj;

struct ns2d_h5_file {
    FILE* fp;
    uint64_t eof;
    h5_obj* root;
    char err[512];
};

static char g_create_err[512];

static int failf(ns2d_h5_file* f, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(f ? f->err : g_create_err, sizeof(g_create_err), fmt, ap);
    va_end(ap);
    return -1;
}

/* ---- growable little-endian byte buffer ---------------------------------- */
typedef struct buf {
    unsigned char* p;
    size_t n, cap;
} buf;

static int b_reserve(buf* b, size_t extra) {
    if (b->n + extra <= b->cap) return 0;
    size_t cap = b->cap ? b->cap : 256;
    while (cap < b->n + extra) cap *= 2;
    unsigned char* q = (unsigned char*)realloc(b->p, cap);
    if (!q) return -1;
    b->p = q;
    b->cap = cap;
    return 0;
}
static int b_bytes(buf* b, const void* src, size_t n) {
    if (b_reserve(b, n)) return -1;
    if (src)
        memcpy(b->p + b->n, src, n);
    else
        memset(b->p + b->n, 0, n);
    b->n += n;
    return 0;
}
/* nbytes little-endian bytes of v; bytes beyond the eighth are zero. */
static int b_uint(buf* b, uint64_t v, int nbytes) {
    unsigned char t[8];
    const int n = nbytes < 8 ? nbytes : 8;
    for (int i = 0; i < n; ++i) t[i] = (unsigned char)(v >> (8 * i));
    if (b_bytes(b, t, (size_t)n)) return -1;
    return nbytes > 8 ? b_bytes(b, NULL, (size_t)(nbytes - 8)) : 0;
}
static int b_pad8(buf* b) {
    size_t r = b->n % 8;
    return r ? b_bytes(b, NULL, 8 - r) : 0;
}
static void b_set_uint(buf* b, size_t at, uint64_t v, int nbytes) {
    for (int i = 0; i < nbytes; ++i) b->p[at + i] = (unsigned char)(v >> (8 * i));
}

/* ---- file I/O -------------------------------------------------------------- */
static int write_at(ns2d_h5_file* f, uint64_t addr, const void* p, size_t n) {
    if (fseeko(f->fp, (off_t)addr, SEEK_SET) != 0) return failf(f, "seek failed: %s", strerror(errno));
    if (n && fwrite(p, 1, n, f->fp) != n) return failf(f, "write failed: %s", strerror(errno));
    return 0;
}
/* Append n bytes at the end of the file; *addr receives their address. */
static int append(ns2d_h5_file* f, const void* p, size_t n, uint64_t* addr) {
    *addr = f->eof;
    if (write_at(f, f->eof, p, n)) return -1;
    f->eof += n;
    return 0;
}

/* ---- object tree --------------------------------------------------------- */
static h5_obj* obj_new(int is_group, const char* name) {
    h5_obj* o = (h5_obj*)calloc(1, sizeof(h5_obj));
    if (!o) return NULL;
    o->is_group = is_group;
    o->name = strdup(name);
    if (!o->name) {
        free(o);
        return NULL;
    }
    return o;
}
static void obj_free(h5_obj* o) {
    if (!o) return;
    for (int i = 0; i < o->nkids; ++i) obj_free(o->kids[i]);
    for (int i = 0; i < o->nattrs; ++i) free(o->attrs[i].name);
    free(o->kids);
    free(o->attrs);
    free(o->name);
    free(o);
}
static h5_obj* find_kid(const h5_obj* g, const char* name, size_t len) {
    for (int i = 0; i < g->nkids; ++i)
        if (strlen(g->kids[i]->name) == len && memcmp(g->kids[i]->name, name, len) == 0) return g->kids[i];
    return NULL;
}
static int add_kid(h5_obj* g, h5_obj* k) {
    if (g->nkids == g->capkids) {
        int cap = g->capkids ? 2 * g->capkids : 8;
        h5_obj** q = (h5_obj**)realloc(g->kids, sizeof(h5_obj*) * (size_t)cap);
        if (!q) return -1;
        g->kids = q;
        g->capkids = cap;
    }
    g->kids[g->nkids++] = k;
    return 0;
}

/* Resolve an absolute or root-relative path.  With want_parent, returns the
   parent group and the final component in *leaf / *leaf_len. */
static h5_obj* resolve(ns2d_h5_file* f, const char* path, int want_parent, const char** leaf, size_t* leaf_len) {
    h5_obj* cur = f->root;
    const char* s = path;
    while (*s == '/') ++s;
    if (!*s) {
        if (want_parent) return NULL;
        return cur;
    }
    for (;;) {
        const char* e = strchr(s, '/');
        size_t len = e ? (size_t)(e - s) : strlen(s);
        const char* nxt = e;
        while (nxt && *nxt == '/') ++nxt;
        int last = !nxt || !*nxt;
        if (last && want_parent) {
            *leaf = s;
            *leaf_len = len;
            return cur;
        }
        if (!cur->is_group) return NULL;
        h5_obj* k = find_kid(cur, s, len);
        if (!k) return NULL;
        cur = k;
        if (last) return cur;
        s = nxt;
    }
}

/* ---- public API -------------------------------------------------------------- */
ns2d_h5_file* ns2d_h5_create(const char* path) {
    if (!path) {
        failf(NULL, "null path");
        return NULL;
    }
    ns2d_h5_file* f = (ns2d_h5_file*)calloc(1, sizeof(ns2d_h5_file));
    if (!f) {
        failf(NULL, "out of memory");
        return NULL;
    }
    f->fp = fopen(path, "w+b");
    if (!f->fp) {
        failf(NULL, "cannot create %s: %s", path, strerror(errno));
        free(f);
        return NULL;
    }
    f->root = obj_new(1, "");
    unsigned char zero[SB_SIZE] = {0};
    if (!f->root || write_at(f, 0, zero, SB_SIZE)) {
        failf(NULL, "cannot initialise %s", path);
        if (f->root) obj_free(f->root);
        fclose(f->fp);
        free(f);
        return NULL;
    }
    f->eof = SB_SIZE;
    return f;
}

const char* ns2d_h5_error(const ns2d_h5_file* f) { return f ? f->err : g_create_err; }

int ns2d_h5_exists(ns2d_h5_file* f, const char* path) {
    if (!f || !path) return 0;
    const char* leaf;
    size_t len;
    h5_obj* parent = resolve(f, path, 1, &leaf, &len);
    if (!parent) {
        const char* s = path;
        while (*s == '/') ++s;
        return *s ? 0 : 1; /* "/" is the root */
    }
    return parent->is_group && find_kid(parent, leaf, len) != NULL;
}

static int check_name(ns2d_h5_file* f, const char* leaf, size_t len) {
    if (len == 0) return failf(f, "empty link name");
    if (len > 65535) return failf(f, "link name too long");
    if (len == 1 && leaf[0] == '.') return failf(f, "'.' is not a valid link name");
    return 0;
}

int ns2d_h5_group(ns2d_h5_file* f, const char* path) {
    if (!f || !path) return -1;
    const char* leaf;
    size_t len;
    h5_obj* parent = resolve(f, path, 1, &leaf, &len);
    if (!parent || !parent->is_group) return failf(f, "parent group of %s does not exist", path);
    if (check_name(f, leaf, len)) return -1;
    h5_obj* k = find_kid(parent, leaf, len);
    if (k) return k->is_group ? 0 : failf(f, "%s exists and is a dataset", path);
    char* nm = strndup(leaf, len);
    if (!nm) return failf(f, "out of memory");
    h5_obj* g = obj_new(1, nm);
    free(nm);
    if (!g || add_kid(parent, g)) {
        obj_free(g);
        return failf(f, "out of memory");
    }
    return 0;
}

int ns2d_h5_attr_double(ns2d_h5_file* f, const char* path, const char* name, double value) {
    if (!f || !path || !name || !*name) return -1;
    h5_obj* o = resolve(f, path, 0, NULL, NULL);
    if (!o) return failf(f, "no object at %s", path);
    for (int i = 0; i < o->nattrs; ++i)
        if (strcmp(o->attrs[i].name, name) == 0) return failf(f, "attribute %s exists on %s", name, path);
    if (o->nattrs == o->capattrs) {
        int cap = o->capattrs ? 2 * o->capattrs : 4;
        h5_attr* q = (h5_attr*)realloc(o->attrs, sizeof(h5_attr) * (size_t)cap);
        if (!q) return failf(f, "out of memory");
        o->attrs = q;
        o->capattrs = cap;
    }
    o->attrs[o->nattrs].name = strdup(name);
    if (!o->attrs[o->nattrs].name) return failf(f, "out of memory");
    o->attrs[o->nattrs].value = value;
    o->nattrs++;
    return 0;
}

static size_t type_size(int type) { return type == NS2D_H5_F64 ? 8 : type == NS2D_H5_I32 ? 4 : 16; }

int ns2d_h5_dataset(ns2d_h5_file* f, const char* path, int type, int rank, const uint64_t* dims, const void* data) {
    if (!f || !path || !dims || rank < 1 || rank > 8) return failf(f, "invalid dataset arguments");
    if (type != NS2D_H5_F64 && type != NS2D_H5_I32 && type != NS2D_H5_C128) return failf(f, "unknown type %d", type);
    const char* leaf;
    size_t len;
    h5_obj* parent = resolve(f, path, 1, &leaf, &len);
    if (!parent || !parent->is_group) return failf(f, "parent group of %s does not exist", path);
    if (check_name(f, leaf, len)) return -1;
    if (find_kid(parent, leaf, len)) return failf(f, "%s exists", path);
    uint64_t n = 1;
    for (int i = 0; i < rank; ++i) n *= dims[i];
    const uint64_t bytes = n * type_size(type);
    if (bytes && !data) return failf(f, "null data for %s", path);
    char* nm = strndup(leaf, len);
    if (!nm) return failf(f, "out of memory");
    h5_obj* d = obj_new(0, nm);
    free(nm);
    if (!d) return failf(f, "out of memory");
    d->type = type;
    d->rank = rank;
    for (int i = 0; i < rank; ++i) d->dims[i] = dims[i];
    d->data_size = bytes;
    d->data_addr = H5_UNDEF;
    if (bytes && append(f, data, (size_t)bytes, &d->data_addr)) {
        obj_free(d);
        return -1;
    }
    if (add_kid(parent, d)) {
        obj_free(d);
        return failf(f, "out of memory");
    }
    return 0;
}

/* ---- messages ------------------------------------------------------------------ */
/* Datatype message bodies (version 1). */
static int dt_double(buf* b) {
    b_uint(b, 0x11, 1);            /* version 1, class 1 (floating point) */
    b_uint(b, 0x20, 1);            /* little-endian, implied mantissa MSB */
    b_uint(b, 63, 1);              /* sign bit location */
    b_uint(b, 0, 1);
    b_uint(b, 8, 4);               /* size */
    b_uint(b, 0, 2);               /* bit offset */
    b_uint(b, 64, 2);              /* precision */
    b_uint(b, 52, 1);              /* exponent location */
    b_uint(b, 11, 1);              /* exponent size */
    b_uint(b, 0, 1);               /* mantissa location */
    b_uint(b, 52, 1);              /* mantissa size */
    return b_uint(b, 1023, 4);     /* exponent bias */
}
static int dt_int32(buf* b) {
    b_uint(b, 0x10, 1);            /* version 1, class 0 (fixed point) */
    b_uint(b, 0x08, 1);            /* little-endian, signed */
    b_uint(b, 0, 2);
    b_uint(b, 4, 4);               /* size */
    b_uint(b, 0, 2);               /* bit offset */
    return b_uint(b, 32, 2);       /* precision */
}
static int dt_complex(buf* b) {
    b_uint(b, 0x16, 1);            /* version 1, class 6 (compound) */
    b_uint(b, 2, 2);               /* number of members */
    b_uint(b, 0, 1);
    b_uint(b, 16, 4);              /* size */
    const char* names[2] = {"r", "i"};
    for (int m = 0; m < 2; ++m) {
        size_t l = strlen(names[m]) + 1;
        b_bytes(b, names[m], l);
        b_bytes(b, NULL, ((l + 7) & ~(size_t)7) - l); /* name padded to a multiple of 8 */
        b_uint(b, 8u * (unsigned)m, 4); /* byte offset of the member */
        b_uint(b, 0, 1);           /* dimensionality */
        b_uint(b, 0, 3);
        b_uint(b, 0, 4);           /* dimension permutation */
        b_uint(b, 0, 4);
        b_uint(b, 0, 16);          /* four dimension sizes */
        dt_double(b);
    }
    return 0;
}
static int dt_body(buf* b, int type) {
    return type == NS2D_H5_F64 ? dt_double(b) : type == NS2D_H5_I32 ? dt_int32(b) : dt_complex(b);
}
static int ds_body(buf* b, int rank, const uint64_t* dims) {
    b_uint(b, 1, 1);               /* version 1 */
    b_uint(b, (uint64_t)rank, 1);
    b_uint(b, 0, 1);               /* no maximum dimensions: equal to the current ones */
    b_uint(b, 0, 1);
    b_uint(b, 0, 4);
    for (int i = 0; i < rank; ++i) b_uint(b, dims[i], 8);
    return 0;
}

/* Append one message (type, body) to an object header under construction. */
static int oh_msg(buf* oh, int* nmsg, int type, const buf* body) {
    size_t sz = (body->n + 7) & ~(size_t)7;
    if (sz > 65535) return -1;
    b_uint(oh, (uint64_t)type, 2);
    b_uint(oh, sz, 2);
    b_uint(oh, 0, 1);              /* flags */
    b_uint(oh, 0, 3);
    b_bytes(oh, body->p, body->n);
    b_bytes(oh, NULL, sz - body->n);
    (*nmsg)++;
    return 0;
}

static int attr_msgs(buf* oh, int* nmsg, const h5_obj* o) {
    for (int i = 0; i < o->nattrs; ++i) {
        buf body = {0}, dt = {0}, ds = {0};
        const uint64_t one = 1;
        dt_double(&dt);
        ds_body(&ds, 1, &one);
        size_t nl = strlen(o->attrs[i].name) + 1;
        b_uint(&body, 1, 1);       /* version 1 */
        b_uint(&body, 0, 1);
        b_uint(&body, nl, 2);
        b_uint(&body, dt.n, 2);
        b_uint(&body, ds.n, 2);
        b_bytes(&body, o->attrs[i].name, nl);
        b_pad8(&body);
        b_bytes(&body, dt.p, dt.n);
        b_pad8(&body);
        b_bytes(&body, ds.p, ds.n);
        b_pad8(&body);
        double v = o->attrs[i].value;
        uint64_t bits;
        memcpy(&bits, &v, 8);
        b_uint(&body, bits, 8);
        int r = oh_msg(oh, nmsg, 0x000C, &body);
        free(body.p);
        free(dt.p);
        free(ds.p);
        if (r) return -1;
    }
    return 0;
}

/* Write an object header made of the message block `msgs` (nmsg messages). */
static int write_oh(ns2d_h5_file* f, const buf* msgs, int nmsg, uint64_t* addr) {
    buf h = {0};
    b_uint(&h, 1, 1);              /* version 1 */
    b_uint(&h, 0, 1);
    b_uint(&h, (uint64_t)nmsg, 2);
    b_uint(&h, 1, 4);              /* reference count */
    b_uint(&h, msgs->n, 4);        /* header data size (messages only) */
    b_uint(&h, 0, 4);              /* alignment of the first message */
    b_bytes(&h, msgs->p, msgs->n);
    int r = h.p ? append(f, h.p, h.n, addr) : -1;
    free(h.p);
    return r;
}

static int flush_dataset(ns2d_h5_file* f, h5_obj* d) {
    buf msgs = {0}, body = {0};
    int nmsg = 0, r = 0;
    ds_body(&body, d->rank, d->dims);
    r |= oh_msg(&msgs, &nmsg, 0x0001, &body);
    body.n = 0;
    dt_body(&body, d->type);
    r |= oh_msg(&msgs, &nmsg, 0x0003, &body);
    body.n = 0;
    b_uint(&body, 2, 1);           /* fill value message version 2 */
    b_uint(&body, 2, 1);           /* allocation time: late */
    b_uint(&body, 2, 1);           /* write time: if set */
    b_uint(&body, 0, 1);           /* no fill value defined */
    r |= oh_msg(&msgs, &nmsg, 0x0005, &body);
    body.n = 0;
    b_uint(&body, 3, 1);           /* layout message version 3 */
    b_uint(&body, 1, 1);           /* contiguous */
    b_uint(&body, d->data_addr, 8);
    b_uint(&body, d->data_size, 8);
    r |= oh_msg(&msgs, &nmsg, 0x0008, &body);
    r |= attr_msgs(&msgs, &nmsg, d);
    if (!r)
        r = write_oh(f, &msgs, nmsg, &d->oh_addr);
    else
        failf(f, "object header of %s too large", d->name);
    free(msgs.p);
    free(body.p);
    return r;
}

static int cmp_kids(const void* a, const void* b) {
    return strcmp((*(h5_obj* const*)a)->name, (*(h5_obj* const*)b)->name);
}

static int flush_obj(ns2d_h5_file* f, h5_obj* o);

static int flush_group(ns2d_h5_file* f, h5_obj* g) {
    for (int i = 0; i < g->nkids; ++i)
        if (flush_obj(f, g->kids[i])) return -1;
    if (g->nkids > 1) qsort(g->kids, (size_t)g->nkids, sizeof(h5_obj*), cmp_kids);
    const int n = g->nkids;
    int rc = -1;
    uint64_t* off = (uint64_t*)calloc((size_t)n + 1, sizeof(uint64_t));
    buf heap = {0}, blk = {0};
    if (!off) return failf(f, "out of memory");

    /* local heap: offset 0 holds the empty name, then the link names */
    b_bytes(&heap, NULL, 8);
    for (int i = 0; i < n; ++i) {
        off[i] = heap.n;
        b_bytes(&heap, g->kids[i]->name, strlen(g->kids[i]->name) + 1);
        b_pad8(&heap);
    }
    b_bytes(&blk, "HEAP", 4);
    b_uint(&blk, 0, 1);            /* version 0 */
    b_uint(&blk, 0, 3);
    b_uint(&blk, heap.n, 8);       /* data segment size */
    b_uint(&blk, 1, 8);            /* free list: none */
    b_uint(&blk, f->eof + 32, 8);  /* data segment follows the header */
    b_bytes(&blk, heap.p, heap.n);
    if (append(f, blk.p, blk.n, &g->heap_addr)) goto out;

    /* symbol-table nodes */
    const int nsnod = (n + SNOD_CAP - 1) / SNOD_CAP;
    const uint64_t snod0 = f->eof;
    for (int s = 0; s < nsnod; ++s) {
        const int lo = s * SNOD_CAP, hi = (lo + SNOD_CAP < n) ? lo + SNOD_CAP : n;
        blk.n = 0;
        b_bytes(&blk, "SNOD", 4);
        b_uint(&blk, 1, 1);        /* version 1 */
        b_uint(&blk, 0, 1);
        b_uint(&blk, (uint64_t)(hi - lo), 2);
        for (int i = lo; i < hi; ++i) {
            b_uint(&blk, off[i], 8);
            b_uint(&blk, g->kids[i]->oh_addr, 8);
            b_uint(&blk, 0, 4);    /* nothing cached */
            b_uint(&blk, 0, 4);
            b_uint(&blk, 0, 16);
        }
        b_bytes(&blk, NULL, SNOD_SIZE - blk.n);
        uint64_t a;
        if (append(f, blk.p, blk.n, &a)) goto out;
    }

    /* B-tree, bottom-up.  Level 0 indexes the SNODs; each higher level
       indexes the level below.  Child c covers names in (key c, key c+1]. */
    {
        int nchild = nsnod;
        uint64_t child0 = snod0, child_stride = SNOD_SIZE;
        /* right key of child c (heap offset of its largest name) */
        uint64_t* rkey = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(nsnod > 0 ? nsnod : 1));
        if (!rkey) {
            failf(f, "out of memory");
            goto out;
        }
        for (int s = 0; s < nsnod; ++s) {
            const int hi = ((s + 1) * SNOD_CAP < n) ? (s + 1) * SNOD_CAP : n;
            rkey[s] = off[hi - 1];
        }
        int level = 0;
        for (;;) {
            const int nnodes = nchild <= BT_CAP ? 1 : (nchild + BT_CAP - 1) / BT_CAP;
            const uint64_t base = f->eof;
            uint64_t* nrkey = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)nnodes);
            if (!nrkey) {
                free(rkey);
                failf(f, "out of memory");
                goto out;
            }
            for (int k = 0; k < nnodes; ++k) {
                const int lo = k * BT_CAP, hi = (lo + BT_CAP < nchild) ? lo + BT_CAP : nchild;
                blk.n = 0;
                b_bytes(&blk, "TREE", 4);
                b_uint(&blk, 0, 1);   /* node type 0: group nodes */
                b_uint(&blk, (uint64_t)level, 1);
                b_uint(&blk, (uint64_t)(hi - lo), 2);
                b_uint(&blk, k > 0 ? base + (uint64_t)(k - 1) * BT_SIZE : H5_UNDEF, 8);
                b_uint(&blk, k + 1 < nnodes ? base + (uint64_t)(k + 1) * BT_SIZE : H5_UNDEF, 8);
                b_uint(&blk, lo > 0 ? rkey[lo - 1] : 0, 8); /* left key */
                for (int c = lo; c < hi; ++c) {
                    b_uint(&blk, child0 + (uint64_t)c * child_stride, 8);
                    b_uint(&blk, rkey[c], 8);
                }
                b_bytes(&blk, NULL, BT_SIZE - blk.n);
                nrkey[k] = hi > lo ? rkey[hi - 1] : 0;
                uint64_t a;
                if (append(f, blk.p, blk.n, &a)) {
                    free(rkey);
                    free(nrkey);
                    goto out;
                }
            }
            free(rkey);
            rkey = nrkey;
            if (nnodes == 1) {
                g->btree_addr = base;
                break;
            }
            nchild = nnodes;
            child0 = base;
            child_stride = BT_SIZE;
            ++level;
        }
        free(rkey);
    }

    /* the group's object header: symbol table message + attributes */
    {
        buf msgs = {0}, body = {0};
        int nmsg = 0;
        b_uint(&body, g->btree_addr, 8);
        b_uint(&body, g->heap_addr, 8);
        int r = oh_msg(&msgs, &nmsg, 0x0011, &body);
        r |= attr_msgs(&msgs, &nmsg, g);
        if (!r)
            r = write_oh(f, &msgs, nmsg, &g->oh_addr);
        else
            failf(f, "object header of group %s too large", g->name);
        free(msgs.p);
        free(body.p);
        if (r) goto out;
    }
    rc = 0;
out:
    free(off);
    free(heap.p);
    free(blk.p);
    return rc;
}

static int flush_obj(ns2d_h5_file* f, h5_obj* o) { return o->is_group ? flush_group(f, o) : flush_dataset(f, o); }

int ns2d_h5_flush(ns2d_h5_file* f) {
    if (!f) return -1;
    if (flush_group(f, f->root)) return -1;
    buf sb = {0};
    static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    b_bytes(&sb, sig, 8);
    b_uint(&sb, 0, 1);             /* superblock version 0 */
    b_uint(&sb, 0, 1);             /* free-space storage version */
    b_uint(&sb, 0, 1);             /* root group symbol table entry version */
    b_uint(&sb, 0, 1);
    b_uint(&sb, 0, 1);             /* shared header message format version */
    b_uint(&sb, 8, 1);             /* size of offsets */
    b_uint(&sb, 8, 1);             /* size of lengths */
    b_uint(&sb, 0, 1);
    b_uint(&sb, LEAF_K, 2);
    b_uint(&sb, NODE_K, 2);
    b_uint(&sb, 0, 4);             /* file consistency flags */
    b_uint(&sb, 0, 8);             /* base address */
    b_uint(&sb, H5_UNDEF, 8);      /* free-space info */
    const size_t eof_at = sb.n;
    b_uint(&sb, 0, 8);             /* end of file address (below) */
    b_uint(&sb, H5_UNDEF, 8);      /* driver information block */
    b_uint(&sb, 0, 8);             /* root entry: link name offset */
    b_uint(&sb, f->root->oh_addr, 8);
    b_uint(&sb, 1, 4);             /* cache type 1: symbol table addresses cached */
    b_uint(&sb, 0, 4);
    b_uint(&sb, f->root->btree_addr, 8);
    b_uint(&sb, f->root->heap_addr, 8);
    b_set_uint(&sb, eof_at, f->eof, 8);
    int r = (sb.n == SB_SIZE) ? write_at(f, 0, sb.p, sb.n) : failf(f, "superblock size %zu", sb.n);
    free(sb.p);
    if (!r && fflush(f->fp) != 0) r = failf(f, "flush failed: %s", strerror(errno));
    return r;
}

int ns2d_h5_close(ns2d_h5_file* f) {
    if (!f) return -1;
    int r = ns2d_h5_flush(f);
    if (fclose(f->fp) != 0) r = -1;
    if (r) snprintf(g_create_err, sizeof(g_create_err), "%s", f->err);
    obj_free(f->root);
    free(f);
    return r;
}

/* ---- reading ------------------------------------------------------------------ */
/* Reader for files in libhdf5's default layout, for input files (MAX_PALIN,
   Solver/src/solver.c:1775-1853) and for post-processing saved runs
   (PostProcessing/src/hdf5_funcs.c:33-170): superblock version 0 or 1 with
   8-byte offsets and lengths, version-1 object headers (with continuation
   blocks), symbol-table groups, datasets of IEEE little-endian doubles, 32-bit
   little-endian ints or the {r, i} compound of two doubles, contiguous or
   compact layout (message version 3), version-1 attributes of one double.
   Other layouts are reported as unsupported.  Each call opens the file, finds
   its object and closes it again. */
typedef struct h5_in {
    FILE* fp;
    uint64_t size;
    int leaf_k, node_k;
    uint64_t root_oh;
} h5_in;

static int rd(h5_in* in, uint64_t addr, void* dst, size_t n) {
    if (addr > in->size || n > in->size - addr)
        return failf(NULL, "read beyond end of file at %llu", (unsigned long long)addr);
    if (fseeko(in->fp, (off_t)addr, SEEK_SET) != 0 || fread(dst, 1, n, in->fp) != n) return failf(NULL, "read failed");
    return 0;
}
static uint64_t le(const unsigned char* p, int n) {
    uint64_t v = 0;
    for (int i = n - 1; i >= 0; --i) v = (v << 8) | p[i];
    return v;
}

static int open_in(h5_in* in, const char* path) {
    memset(in, 0, sizeof(*in));
    in->fp = fopen(path, "rb");
    if (!in->fp) return failf(NULL, "cannot open %s: %s", path, strerror(errno));
    unsigned char sb[56], ent[40];
    fseeko(in->fp, 0, SEEK_END);
    in->size = (uint64_t)ftello(in->fp);
    static const unsigned char sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
    if (rd(in, 0, sb, 56) || memcmp(sb, sig, 8) != 0) return failf(NULL, "%s is not an HDF5 file (superblock at 0 only)", path);
    if (sb[8] > 1 || sb[13] != 8 || sb[14] != 8)
        return failf(NULL, "superblock version %d / offset size %d unsupported", sb[8], sb[13]);
    in->leaf_k = (int)le(sb + 16, 2);
    in->node_k = (int)le(sb + 18, 2);
    if (in->leaf_k <= 0 || in->node_k <= 0 || rd(in, sb[8] == 0 ? 56 : 60, ent, 40)) return failf(NULL, "bad superblock");
    in->root_oh = le(ent + 8, 8);
    return 0;
}

/* Messages of the v1 object header at addr: calls fn(ctx, type, body, size). */
typedef int (*msg_fn)(void* ctx, int type, const unsigned char* body, size_t size);
static int walk_header(h5_in* in, uint64_t addr, msg_fn fn, void* ctx) {
    unsigned char pre[16];
    if (rd(in, addr, pre, 16)) return -1;
    if (pre[0] != 1) return failf(NULL, "object header version %d unsupported", pre[0]);
    uint64_t chunk = addr + 16, len = le(pre + 8, 4);
    int budget = 64;
    while (len && budget-- > 0) {
        if (len > in->size) return failf(NULL, "object header block too large");
        unsigned char* c = (unsigned char*)malloc((size_t)len);
        if (!c) return failf(NULL, "out of memory");
        if (rd(in, chunk, c, (size_t)len)) {
            free(c);
            return -1;
        }
        uint64_t next = 0, next_len = 0;
        size_t at = 0;
        while (at + 8 <= len) {
            const int type = (int)le(c + at, 2);
            const size_t sz = (size_t)le(c + at + 2, 2);
            if (at + 8 + sz > len) {
                free(c);
                return failf(NULL, "object header message overruns its block");
            }
            if (type == 0x10 && sz >= 16) {
                next = le(c + at + 8, 8);
                next_len = le(c + at + 16, 8);
            } else if (fn(ctx, type, c + at + 8, sz)) {
                free(c);
                return -1;
            }
            at += 8 + sz;
        }
        free(c);
        chunk = next;
        len = next_len;
    }
    return 0;
}

/* Element type (NS2D_H5_*) of the datatype message at b, or -1. */
static int is_ieee_double(const unsigned char* b, size_t n) {
    return n >= 20 && (b[0] & 0x0f) == 1 && le(b + 4, 4) == 8 && !(b[1] & 1) && le(b + 10, 2) == 64 && b[12] == 52 &&
           b[13] == 11 && b[15] == 52 && le(b + 16, 4) == 1023;
}
static int dtype_code(const unsigned char* b, size_t n) {
    if (n < 8) return -1;
    const int cls = b[0] & 0x0f, ver = b[0] >> 4;
    const uint64_t size = le(b + 4, 4);
    if (is_ieee_double(b, n)) return NS2D_H5_F64;
    if (cls == 0 && size == 4 && n >= 12 && !(b[1] & 1) && (b[1] & 8) && le(b + 10, 2) == 32) return NS2D_H5_I32;
    if (cls == 6 && size == 16 && le(b + 1, 2) == 2 && (ver == 1 || ver == 3)) {
        size_t p = 8;
        const char* names[2] = {"r", "i"};
        for (int m = 0; m < 2; ++m) {
            const size_t l = strlen(names[m]) + 1;
            if (p + l > n || memcmp(b + p, names[m], l) != 0) return -1;
            uint64_t off;
            if (ver == 1) {
                p += (l + 7) & ~(size_t)7;
                if (p + 32 > n) return -1;
                off = le(b + p, 4);
                p += 32;
            } else {
                p += l;
                if (p + 1 > n) return -1;
                off = b[p];
                p += 1;
            }
            if (off != 8u * (unsigned)m || !is_ieee_double(b + p, n - p)) return -1;
            p += 20;
        }
        return NS2D_H5_C128;
    }
    return -1;
}

typedef struct obj_info {
    uint64_t btree, heap;
    int is_group, type, rank;
    uint64_t dims[8], count;
    int layout; /* 1 contiguous, 0 compact, -1 none */
    uint64_t data_addr, data_size;
    unsigned char compact[4096];
    size_t compact_size;
    const char* want_attr; /* attribute wanted, if any */
    int attr_found;
    double attr_value;
} obj_info;

static int dataspace(const unsigned char* b, size_t n, int* rank, uint64_t* dims, uint64_t* count) {
    if (n < 8) return failf(NULL, "dataspace message unsupported");
    const int ver = b[0], r = b[1];
    const size_t at = ver == 1 ? 8 : 4;
    if ((ver != 1 && ver != 2) || r > 8 || at + 8 * (size_t)r > n) return failf(NULL, "dataspace message unsupported");
    *rank = r;
    *count = 1;
    for (int i = 0; i < r; ++i) {
        dims[i] = le(b + at + 8 * i, 8);
        *count *= dims[i];
    }
    return 0;
}

static int info_fn(void* ctx, int type, const unsigned char* b, size_t n) {
    obj_info* o = (obj_info*)ctx;
    if (type == 0x11 && n >= 16) {
        o->is_group = 1;
        o->btree = le(b, 8);
        o->heap = le(b + 8, 8);
    } else if (type == 0x01) {
        return dataspace(b, n, &o->rank, o->dims, &o->count);
    } else if (type == 0x03) {
        o->type = dtype_code(b, n);
    } else if (type == 0x08 && n >= 2) {
        if (b[0] != 3) return failf(NULL, "layout message version %d unsupported", b[0]);
        if (b[1] == 1 && n >= 18) {
            o->layout = 1;
            o->data_addr = le(b + 2, 8);
            o->data_size = le(b + 10, 8);
        } else if (b[1] == 0 && n >= 4) {
            const size_t cs = (size_t)le(b + 2, 2);
            if (4 + cs > n || cs > sizeof(o->compact)) return failf(NULL, "compact dataset too large");
            o->layout = 0;
            memcpy(o->compact, b + 4, cs);
            o->compact_size = cs;
        } else {
            return failf(NULL, "chunked or virtual datasets unsupported");
        }
    } else if (type == 0x0C && o->want_attr && n >= 8 && b[0] == 1) {
        const size_t nl = (size_t)le(b + 2, 2), dl = (size_t)le(b + 4, 2), sl = (size_t)le(b + 6, 2);
        size_t p = 8;
        if (p + nl > n || nl == 0 || b[p + nl - 1] != 0) return 0;
        const int match = strcmp((const char*)b + p, o->want_attr) == 0;
        p += (nl + 7) & ~(size_t)7;
        if (!match || p + dl > n) return 0;
        const int dt = is_ieee_double(b + p, dl) ? NS2D_H5_F64 : -1;
        p += (dl + 7) & ~(size_t)7;
        int r;
        uint64_t dims[8], cnt;
        if (p + sl > n || dataspace(b + p, sl, &r, dims, &cnt)) return -1;
        p += (sl + 7) & ~(size_t)7;
        if (dt != NS2D_H5_F64 || cnt != 1 || p + 8 > n) return failf(NULL, "attribute %s is not one double", o->want_attr);
        memcpy(&o->attr_value, b + p, 8);
        o->attr_found = 1;
    }
    return 0;
}

/* Visit the links of the symbol-table group (btree, heap): fn(ctx, name,
   header address) returns nonzero to stop (1 = found, -1 = error). */
typedef int (*link_fn)(void* ctx, const char* name, uint64_t oh);
static int walk_btree(h5_in* in, uint64_t btree, const char* names, uint64_t hsize, link_fn fn, void* ctx, int depth) {
    if (depth > 16) return failf(NULL, "B-tree too deep");
    const size_t bt_size = 24 + (size_t)(2 * in->node_k + 1) * 8 + (size_t)(2 * in->node_k) * 8;
    unsigned char* node = (unsigned char*)malloc(bt_size);
    if (!node) return failf(NULL, "out of memory");
    int rc = 0;
    if (rd(in, btree, node, bt_size) || memcmp(node, "TREE", 4) != 0 || node[4] != 0) {
        free(node);
        return failf(NULL, "bad group B-tree");
    }
    const int level = node[5], used = (int)le(node + 6, 2);
    if (used > 2 * in->node_k) {
        free(node);
        return failf(NULL, "bad group B-tree");
    }
    const size_t sn_size = 8 + (size_t)(2 * in->leaf_k) * 40;
    for (int c = 0; c < used && rc == 0; ++c) {
        const uint64_t child = le(node + 24 + 8 + 16 * (size_t)c, 8);
        if (level > 0) {
            rc = walk_btree(in, child, names, hsize, fn, ctx, depth + 1);
            continue;
        }
        unsigned char* sn = (unsigned char*)malloc(sn_size);
        if (!sn || rd(in, child, sn, sn_size) || memcmp(sn, "SNOD", 4) != 0) {
            free(sn);
            rc = failf(NULL, "bad symbol-table node");
            break;
        }
        const int ns = (int)le(sn + 6, 2);
        for (int e = 0; e < ns && e < 2 * in->leaf_k && rc == 0; ++e) {
            const uint64_t off = le(sn + 8 + 40 * (size_t)e, 8);
            if (off < hsize) rc = fn(ctx, names + off, le(sn + 8 + 40 * (size_t)e + 8, 8));
        }
        free(sn);
    }
    free(node);
    return rc;
}
static int walk_group(h5_in* in, uint64_t btree, uint64_t heap, link_fn fn, void* ctx) {
    unsigned char hh[32];
    if (rd(in, heap, hh, 32) || memcmp(hh, "HEAP", 4) != 0) return failf(NULL, "bad local heap");
    const uint64_t hsize = le(hh + 8, 8), haddr = le(hh + 24, 8);
    if (hsize > in->size) return failf(NULL, "bad local heap");
    char* names = (char*)malloc((size_t)hsize + 1);
    if (!names) return failf(NULL, "out of memory");
    int rc = rd(in, haddr, names, (size_t)hsize);
    if (!rc) {
        names[hsize] = '\0';
        rc = walk_btree(in, btree, names, hsize, fn, ctx, 0);
    }
    free(names);
    return rc;
}

typedef struct find_ctx {
    const char* name;
    size_t len;
    uint64_t oh;
} find_ctx;
static int find_fn(void* ctx, const char* name, uint64_t oh) {
    find_ctx* f = (find_ctx*)ctx;
    if (strlen(name) == f->len && memcmp(name, f->name, f->len) == 0) {
        f->oh = oh;
        return 1;
    }
    return 0;
}

/* Header address of the object at `path`: 0 found, 1 absent, -1 error. */
static int locate(h5_in* in, const char* path, uint64_t* oh) {
    *oh = in->root_oh;
    const char* s = path;
    for (;;) {
        while (*s == '/') ++s;
        if (!*s) return 0;
        const char* e = strchr(s, '/');
        const size_t len = e ? (size_t)(e - s) : strlen(s);
        obj_info gi;
        memset(&gi, 0, sizeof(gi));
        gi.layout = -1;
        if (walk_header(in, *oh, info_fn, &gi)) return -1;
        if (!gi.is_group) return 1;
        find_ctx fc = {s, len, 0};
        const int r = walk_group(in, gi.btree, gi.heap, find_fn, &fc);
        if (r < 0) return -1;
        if (r == 0) return 1;
        *oh = fc.oh;
        s += len;
    }
}

static int object_info(const char* path, const char* name, obj_info* oi, h5_in* in) {
    if (!path || !name) return failf(NULL, "invalid arguments");
    if (open_in(in, path)) {
        if (in->fp) fclose(in->fp);
        return -1;
    }
    uint64_t oh;
    const int f = locate(in, name, &oh);
    if (f) {
        if (f > 0) failf(NULL, "%s has no object %s", path, name);
        fclose(in->fp);
        return -1;
    }
    if (walk_header(in, oh, info_fn, oi)) {
        fclose(in->fp);
        return -1;
    }
    return 0;
}

int ns2d_h5_dataset_info(const char* path, const char* dataset, int* type, int* rank, uint64_t* dims) {
    h5_in in;
    obj_info* oi = (obj_info*)calloc(1, sizeof(obj_info));
    if (!oi) return failf(NULL, "out of memory");
    oi->layout = -1;
    oi->type = -1;
    int rc = object_info(path, dataset, oi, &in);
    if (!rc) {
        fclose(in.fp);
        if (oi->is_group || oi->layout < 0) {
            rc = failf(NULL, "%s:%s is not a dataset", path, dataset);
        } else {
            if (type) *type = oi->type;
            if (rank) *rank = oi->rank;
            if (dims)
                for (int i = 0; i < oi->rank; ++i) dims[i] = oi->dims[i];
        }
    }
    free(oi);
    return rc;
}

int ns2d_h5_read(const char* path, const char* dataset, int type, void* out, uint64_t count) {
    h5_in in;
    if (!out) return failf(NULL, "invalid arguments");
    obj_info* oi = (obj_info*)calloc(1, sizeof(obj_info));
    if (!oi) return failf(NULL, "out of memory");
    oi->layout = -1;
    oi->type = -1;
    int rc = object_info(path, dataset, oi, &in);
    if (rc) {
        free(oi);
        return rc;
    }
    const uint64_t bytes = count * type_size(type);
    rc = -1;
    if (oi->type != type || oi->type < 0)
        failf(NULL, "%s:%s does not hold elements of type %d", path, dataset, type);
    else if (oi->count != count)
        failf(NULL, "%s:%s holds %llu values, %llu expected", path, dataset, (unsigned long long)oi->count,
              (unsigned long long)count);
    else if (oi->layout == 1 && oi->data_size == bytes)
        rc = rd(&in, oi->data_addr, out, (size_t)bytes);
    else if (oi->layout == 0 && oi->compact_size == bytes) {
        memcpy(out, oi->compact, (size_t)bytes);
        rc = 0;
    } else
        failf(NULL, "%s:%s: no readable storage", path, dataset);
    fclose(in.fp);
    free(oi);
    return rc;
}

int ns2d_h5_read_double(const char* path, const char* dataset, double* out, uint64_t count) {
    return ns2d_h5_read(path, dataset, NS2D_H5_F64, out, count);
}

int ns2d_h5_read_attr_double(const char* path, const char* object, const char* name, double* value) {
    h5_in in;
    if (!name || !value) return failf(NULL, "invalid arguments");
    obj_info* oi = (obj_info*)calloc(1, sizeof(obj_info));
    if (!oi) return failf(NULL, "out of memory");
    oi->layout = -1;
    oi->want_attr = name;
    int rc = object_info(path, object, oi, &in);
    if (!rc) {
        fclose(in.fp);
        if (oi->attr_found)
            *value = oi->attr_value;
        else
            rc = failf(NULL, "%s:%s has no attribute %s", path, object, name);
    }
    free(oi);
    return rc;
}

typedef struct list_ctx {
    char* buf;
    size_t cap, used;
    int n;
} list_ctx;
static int list_fn(void* ctx, const char* name, uint64_t oh) {
    (void)oh;
    list_ctx* l = (list_ctx*)ctx;
    const size_t len = strlen(name);
    if (l->used + len + 1 > l->cap) return failf(NULL, "name buffer too small");
    memcpy(l->buf + l->used, name, len);
    l->buf[l->used + len] = '\n';
    l->used += len + 1;
    l->n++;
    return 0;
}

int ns2d_h5_list(const char* path, const char* group, char* buf, size_t cap) {
    h5_in in;
    if (!buf || cap == 0) return failf(NULL, "invalid arguments");
    obj_info* oi = (obj_info*)calloc(1, sizeof(obj_info));
    if (!oi) return failf(NULL, "out of memory");
    oi->layout = -1;
    int rc = object_info(path, group, oi, &in);
    if (rc) {
        free(oi);
        return rc;
    }
    list_ctx l = {buf, cap - 1, 0, 0};
    if (!oi->is_group)
        rc = failf(NULL, "%s:%s is not a group", path, group);
    else if (walk_group(&in, oi->btree, oi->heap, list_fn, &l) != 0)
        rc = -1;
    buf[l.used] = '\0';
    fclose(in.fp);
    free(oi);
    return rc ? -1 : l.n;
}
