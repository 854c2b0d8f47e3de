/*
 * oracle/shim/h5log.c -- bodies of the HDF5 stand-in (oracle/shim/hdf5.h,
 * hdf5_hl.h).  Test infrastructure only.
 *
 * Each "HDF5 file" the reference creates becomes a log at the same path:
 *   "NS2DLOG1", then records (native little-endian fields):
 *     u32 kind (1 group, 2 attribute, 3 dataset), u32 len, path[len]
 *     attribute: u32 len, name[len], f64 value
 *     dataset:   u32 type (0 f64, 1 i32, 2 complex {r,i}), u32 rank,
 *                u64 dims[rank], u64 nbytes, data[nbytes] (C order)
 * H5Dwrite gathers the selected hyperslab of the memory space (the padded
 * real arrays of hdf5_funcs.c:1232-1326) into C order; with one rank the file
 * selection is always the whole dataset.  tests/h5log.py reads the log.
 * H5Fopen for reading (MAX_PALIN input) is not supported and fails.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hdf5.h"
#include "hdf5_hl.h"

enum { K_FREE = 0, K_FILE, K_GROUP, K_SPACE, K_DSET, K_ATTR, K_TYPE, K_PLIST };

typedef struct obj {
    int kind;
    hid_t file;      /* owning file id (groups, datasets, attributes) */
    char path[1024]; /* file: its name; others: absolute path in the file */
    char name[128];  /* attribute name */
    FILE* fp;        /* files */
    int rank;
    hsize_t dims[8], start[8], count[8];
    int type; /* 0 f64, 1 i32, 2 compound */
    size_t tsize;
} obj;

#define MAX_OBJ 4096
#define ID0 1000
static obj g_obj[MAX_OBJ];

/* groups created so far, per file name (H5Lexists after reopening) */
typedef struct gname {
    char file[1024];
    char path[1024];
} gname;
static gname* g_groups;
static int g_ngroups, g_capgroups;

static hid_t new_obj(int kind) {
    for (int i = 0; i < MAX_OBJ; ++i)
        if (g_obj[i].kind == K_FREE) {
            memset(&g_obj[i], 0, sizeof(obj));
            g_obj[i].kind = kind;
            return ID0 + i;
        }
    return -1;
}
static obj* get(hid_t id, int kind) {
    if (id < ID0 || id >= ID0 + MAX_OBJ) return NULL;
    obj* o = &g_obj[id - ID0];
    return (o->kind == kind || (kind == -1 && o->kind != K_FREE)) ? o : NULL;
}
static void release(hid_t id) {
    obj* o = get(id, -1);
    if (o) o->kind = K_FREE;
}

static const char* loc_path(hid_t loc, hid_t* file) {
    if (get(loc, K_FILE)) {
        *file = loc;
        return "";
    }
    obj* g = get(loc, K_GROUP);
    if (g) {
        *file = g->file;
        return g->path;
    }
    *file = -1;
    return NULL;
}
static void join(char* out, size_t cap, const char* base, const char* name) {
    if (name[0] == '/')
        snprintf(out, cap, "%s", name);
    else
        snprintf(out, cap, "%s/%s", base, name);
}
static void w32(FILE* fp, uint32_t v) { fwrite(&v, 4, 1, fp); }
static void w64(FILE* fp, uint64_t v) { fwrite(&v, 8, 1, fp); }
static void wstr(FILE* fp, const char* s) {
    w32(fp, (uint32_t)strlen(s));
    fwrite(s, 1, strlen(s), fp);
}

hid_t H5Fcreate(const char* name, unsigned flags, hid_t fcpl, hid_t fapl) {
    (void)flags; (void)fcpl; (void)fapl;
    hid_t id = new_obj(K_FILE);
    if (id < 0) return -1;
    obj* f = get(id, K_FILE);
    f->fp = fopen(name, "wb");
    if (!f->fp) {
        release(id);
        return -1;
    }
    snprintf(f->path, sizeof(f->path), "%s", name);
    fwrite("NS2DLOG1", 1, 8, f->fp);
    /* on disk now: with transient iterations the reference never closes this
       handle (hdf5_funcs.c:400-410) and reopens the file to append */
    fflush(f->fp);
    for (int i = 0; i < g_ngroups; ++i)
        if (!strcmp(g_groups[i].file, name)) g_groups[i].file[0] = '\0';
    return id;
}
hid_t H5Fopen(const char* name, unsigned flags, hid_t fapl) {
    (void)fapl;
    if (flags != H5F_ACC_RDWR) return -1;
    hid_t id = new_obj(K_FILE);
    if (id < 0) return -1;
    obj* f = get(id, K_FILE);
    f->fp = fopen(name, "ab");
    if (!f->fp) {
        release(id);
        return -1;
    }
    snprintf(f->path, sizeof(f->path), "%s", name);
    return id;
}
herr_t H5Fclose(hid_t id) {
    obj* f = get(id, K_FILE);
    if (!f) return -1;
    fclose(f->fp);
    release(id);
    return 0;
}
hid_t H5Pcreate(hid_t cls) {
    (void)cls;
    return new_obj(K_PLIST);
}
herr_t H5Pset_fapl_mpio(hid_t p, int comm, int info) { (void)p; (void)comm; (void)info; return 0; }
herr_t H5Pset_dxpl_mpio(hid_t p, int mode) { (void)p; (void)mode; return 0; }
herr_t H5Pclose(hid_t p) {
    release(p);
    return 0;
}

htri_t H5Lexists(hid_t loc, const char* name, hid_t lapl) {
    (void)lapl;
    hid_t file;
    const char* base = loc_path(loc, &file);
    if (!base) return -1;
    char path[1024];
    join(path, sizeof(path), base, name);
    const char* fname = get(file, K_FILE)->path;
    for (int i = 0; i < g_ngroups; ++i)
        if (!strcmp(g_groups[i].file, fname) && !strcmp(g_groups[i].path, path)) return 1;
    return 0;
}
static hid_t open_group(hid_t loc, const char* name, int create) {
    hid_t file;
    const char* base = loc_path(loc, &file);
    if (!base) return -1;
    hid_t id = new_obj(K_GROUP);
    if (id < 0) return -1;
    obj* g = get(id, K_GROUP);
    g->file = file;
    join(g->path, sizeof(g->path), base, name);
    if (create) {
        obj* f = get(file, K_FILE);
        w32(f->fp, 1);
        wstr(f->fp, g->path);
        if (g_ngroups == g_capgroups) {
            g_capgroups = g_capgroups ? 2 * g_capgroups : 64;
            g_groups = (gname*)realloc(g_groups, sizeof(gname) * (size_t)g_capgroups);
        }
        snprintf(g_groups[g_ngroups].file, sizeof(g_groups[0].file), "%s", f->path);
        snprintf(g_groups[g_ngroups].path, sizeof(g_groups[0].path), "%s", g->path);
        g_ngroups++;
    }
    return id;
}
hid_t H5Gcreate(hid_t loc, const char* name, hid_t lcpl, hid_t gcpl, hid_t gapl) {
    (void)lcpl; (void)gcpl; (void)gapl;
    return open_group(loc, name, 1);
}
hid_t H5Gopen(hid_t loc, const char* name, hid_t gapl) {
    (void)gapl;
    return open_group(loc, name, 0);
}
herr_t H5Gclose(hid_t g) {
    release(g);
    return 0;
}

hid_t H5Screate_simple(int rank, const hsize_t* dims, const hsize_t* maxdims) {
    (void)maxdims;
    if (rank < 1 || rank > 8) return -1;
    hid_t id = new_obj(K_SPACE);
    if (id < 0) return -1;
    obj* s = get(id, K_SPACE);
    s->rank = rank;
    for (int i = 0; i < rank; ++i) {
        s->dims[i] = dims[i];
        s->start[i] = 0;
        s->count[i] = dims[i];
    }
    return id;
}
herr_t H5Sselect_hyperslab(hid_t space, int op, const hsize_t* start, const hsize_t* stride, const hsize_t* count,
                           const hsize_t* block) {
    (void)op;
    obj* s = get(space, K_SPACE);
    if (!s || stride || block) return -1;
    for (int i = 0; i < s->rank; ++i) {
        if (start[i] + count[i] > s->dims[i]) return -1;
        s->start[i] = start[i];
        s->count[i] = count[i];
    }
    return 0;
}
herr_t H5Sclose(hid_t s) {
    release(s);
    return 0;
}

static int type_code(hid_t t, size_t* size) {
    if (t == H5T_NATIVE_DOUBLE) {
        *size = 8;
        return 0;
    }
    if (t == H5T_NATIVE_INT) {
        *size = 4;
        return 1;
    }
    obj* c = get(t, K_TYPE);
    if (c && c->tsize == 16) {
        *size = 16;
        return 2;
    }
    return -1;
}

hid_t H5Tcreate(int cls, size_t size) {
    if (cls != H5T_COMPOUND) return -1;
    hid_t id = new_obj(K_TYPE);
    if (id >= 0) get(id, K_TYPE)->tsize = size;
    return id;
}
herr_t H5Tinsert(hid_t type, const char* name, size_t offset, hid_t member) {
    if (!get(type, K_TYPE) || member != H5T_NATIVE_DOUBLE) return -1;
    if (!((!strcmp(name, "r") && offset == 0) || (!strcmp(name, "i") && offset == 8))) return -1;
    return 0;
}
herr_t H5Tclose(hid_t t) {
    release(t);
    return 0;
}

hid_t H5Dcreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t lcpl, hid_t dcpl, hid_t dapl) {
    (void)lcpl; (void)dcpl; (void)dapl;
    hid_t file;
    const char* base = loc_path(loc, &file);
    obj* s = get(space, K_SPACE);
    size_t tsize;
    const int code = type_code(type, &tsize);
    if (!base || !s || code < 0) return -1;
    hid_t id = new_obj(K_DSET);
    if (id < 0) return -1;
    obj* d = get(id, K_DSET);
    d->file = file;
    join(d->path, sizeof(d->path), base, name);
    d->rank = s->rank;
    for (int i = 0; i < s->rank; ++i) d->dims[i] = s->dims[i];
    d->type = code;
    d->tsize = tsize;
    return id;
}

static void record(obj* f, const char* path, int type, int rank, const hsize_t* dims, const void* data, size_t nbytes) {
    w32(f->fp, 3);
    wstr(f->fp, path);
    w32(f->fp, (uint32_t)type);
    w32(f->fp, (uint32_t)rank);
    for (int i = 0; i < rank; ++i) w64(f->fp, dims[i]);
    w64(f->fp, nbytes);
    fwrite(data, 1, nbytes, f->fp);
}

herr_t H5Dwrite(hid_t dset, hid_t memtype, hid_t memspace, hid_t filespace, hid_t plist, const void* buf) {
    (void)memtype; (void)plist;
    obj* d = get(dset, K_DSET);
    if (!d) return -1;
    size_t n = 1;
    for (int i = 0; i < d->rank; ++i) n *= d->dims[i];
    if (filespace != H5S_ALL) {
        obj* fs = get(filespace, K_SPACE);
        if (!fs) return -1;
        for (int i = 0; i < fs->rank; ++i)
            if (fs->start[i] != 0 || fs->count[i] != d->dims[i]) return -1; /* one rank writes everything */
    }
    unsigned char* out = (unsigned char*)malloc(n * d->tsize + 1);
    if (!out) return -1;
    if (memspace == H5S_ALL) {
        memcpy(out, buf, n * d->tsize);
    } else {
        obj* ms = get(memspace, K_SPACE);
        if (!ms || ms->rank != d->rank) {
            free(out);
            return -1;
        }
        hsize_t idx[8] = {0};
        size_t o = 0;
        for (size_t e = 0; e < n; ++e) {
            size_t off = 0;
            for (int k = 0; k < ms->rank; ++k) off = off * ms->dims[k] + (ms->start[k] + idx[k]);
            memcpy(out + o, (const unsigned char*)buf + off * d->tsize, d->tsize);
            o += d->tsize;
            for (int k = ms->rank - 1; k >= 0; --k) {
                if (++idx[k] < ms->count[k]) break;
                idx[k] = 0;
            }
        }
    }
    record(get(d->file, K_FILE), d->path, d->type, d->rank, d->dims, out, n * d->tsize);
    free(out);
    return 0;
}
herr_t H5Dclose(hid_t d) {
    release(d);
    return 0;
}

hid_t H5Acreate(hid_t loc, const char* name, hid_t type, hid_t space, hid_t acpl, hid_t aapl) {
    (void)space; (void)acpl; (void)aapl;
    hid_t file;
    const char* base = loc_path(loc, &file);
    if (!base || type != H5T_NATIVE_DOUBLE) return -1;
    hid_t id = new_obj(K_ATTR);
    if (id < 0) return -1;
    obj* a = get(id, K_ATTR);
    a->file = file;
    snprintf(a->path, sizeof(a->path), "%s", base[0] ? base : "/");
    snprintf(a->name, sizeof(a->name), "%s", name);
    return id;
}
herr_t H5Awrite(hid_t attr, hid_t type, const void* buf) {
    obj* a = get(attr, K_ATTR);
    if (!a || type != H5T_NATIVE_DOUBLE) return -1;
    obj* f = get(a->file, K_FILE);
    w32(f->fp, 2);
    wstr(f->fp, a->path);
    wstr(f->fp, a->name);
    double v;
    memcpy(&v, buf, 8);
    fwrite(&v, 8, 1, f->fp);
    return 0;
}
herr_t H5Aclose(hid_t a) {
    release(a);
    return 0;
}

herr_t H5LTmake_dataset(hid_t loc, const char* name, int rank, const hsize_t* dims, hid_t type, const void* buf) {
    hid_t file;
    const char* base = loc_path(loc, &file);
    size_t tsize;
    const int code = type_code(type, &tsize);
    if (!base || code < 0 || rank < 1 || rank > 8) return -1;
    char path[1024];
    join(path, sizeof(path), base, name);
    size_t n = 1;
    for (int i = 0; i < rank; ++i) n *= dims[i];
    record(get(file, K_FILE), path, code, rank, dims, buf, n * tsize);
    return 0;
}
herr_t H5LTread_dataset_double(hid_t loc, const char* name, double* buf) {
    (void)loc; (void)name; (void)buf;
    return -1;
}
/* reads are not logged files' business: the callers' error paths follow */
herr_t H5LTread_dataset(hid_t loc, const char* name, hid_t type, void* buf) {
    (void)loc; (void)name; (void)type; (void)buf;
    return -1;
}
