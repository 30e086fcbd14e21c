/*
 * writer.cpp -- output steps in the reference's on-disk formats, and the
 * asynchronous writer that produces them from device snapshots.
 *
 * Formats (AgentBasedModel-BacColonyGrowth/):
 *   directory tree       CreateOutputFiles, InputOutput.cpp:42-271
 *   Cells/<id>.txt       Output, InputOutput.cpp:799-817 (one line per cell)
 *   Restart/<id>.txt     SaveCells, InputOutput.cpp:434-448 ({t, dt, Cell[n]})
 *   Density/<id>.txt     Array3D<double>::Output(f, 1), Array.h:568-584
 *   Environment/<id>.txt Array3D<LocalEnv>::Output(f, 1), Array.h:931-1122
 *   AgarField/<id>.txt   Array3D<LocalAga>::Append(f, 1) per level, Array.h:1447-1494
 *   WallField/<id>.txt   Array2D<LocalAga>::Append(f) per level, Array.h:419-457
 *   lineage/0.txt        CreateOutputFileLineage, InputOutput.cpp:13-33, and
 *                        the "%d %d\n" lines of Simulation.cpp:392
 * Every number goes through the reference's own printf conversion, so a
 * file holds the reference's bytes for the same values.  With Box_y = 1
 * every field file is a sequence of rows of Box_x numbers, one row per z
 * (per member, per level); Density adds an empty line after each row.
 *
 * Formatting is the expensive part (about 30 conversions per cell), so a
 * file is cut into contiguous ranges of lines that are formatted on
 * `threads` threads and written in order.  The asynchronous writer runs
 * this on its own host thread, behind a copy of the step's snapshot into
 * pinned memory, so a simulation thread only pays for queuing the snapshot.
 */
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/bcg.h"
#include "internal.h"

void bcg_set_cuda_error(cudaError_t e);   /* ctx.cu */

namespace {

/* the printf conversions of Output's cell line, InputOutput.cpp:803-805 */
#define CELL_LINE "%4.4f %d %d %4.4f %4.4f %4.4f %4.4f %4.4f %4.4f %4.4f %4.4f %4.4E %4.4E %4.4E %4.4E %4.4E %4.4E " \
                  "%4.4f %4.4f %4.4f %4.4f %4.4f %4.4f %4.4f %4.4f %d %d %d\n"
/* the conversion of every field value, Array.h:568-1494 */
#define FIELD_VALUE "%6E\t"

/* CreateOutputFiles' directories, in its order; all but six stay empty */
const char* const kTree[17] = {"Cells", "Restart", "RoughDensity", "RoughDensity1", "RoughDensity2",
                               "Density", "Density1", "Density2", "WallDensity", "WallDensity1",
                               "WallDensity2", "RoughHeight", "Height", "Normal", "Environment",
                               "AgarField", "WallField"};

/* a field plane: value(x, z) = p[x * sx + z * sz]; a null p reads zeros */
struct Plane { const double* p; ptrdiff_t sx, sz; };
/* one row of a field file: Box_x values of plane row z, then "\n" (and for
 * Array3D<double>::Output, the empty line of its z loop) */
struct Row { Plane pl; int z; bool blank; };

struct Step {
    double t = 0, dt = 0;
    int n_cells = 0, force_stride = 3;
    const bcg_cell* cells = nullptr;
    const double* force = nullptr;
    int n_restart = -1;
    const bcg_cell* restart = nullptr;
    int X = 0, Z = 0, Za = 0, levels = 0;
    Plane density{};
    Plane env[17]{};
    std::vector<Plane> agar;   /* 4 per level: carbon, acetate, waste, oxygen */
    std::vector<Plane> wall;   /* 4 per level */
};

template <class... A>
void appendf(std::string& out, const char* fmt, A... a)
{
    char buf[256];
    int k = snprintf(buf, sizeof buf, fmt, a...);
    if (k < 0) return;
    if ((size_t)k < sizeof buf) { out.append(buf, (size_t)k); return; }
    size_t o = out.size();
    out.resize(o + (size_t)k + 1);
    snprintf(&out[o], (size_t)k + 1, fmt, a...);
    out.resize(o + (size_t)k);
}

/* fn(begin, end, text) over [0, n) cut into at most `threads` contiguous
 * parts of at least min_part items; the parts come back in order */
template <class F>
std::vector<std::string> in_parts(size_t n, int threads, size_t min_part, F fn)
{
    size_t parts = std::min<size_t>((size_t)std::max(threads, 1), (n + min_part - 1) / min_part);
    parts = std::max<size_t>(parts, 1);
    std::vector<std::string> out(parts);
    std::vector<std::thread> pool;
    for (size_t p = 0; p + 1 < parts; p++) {
        size_t b = n * p / parts, e = n * (p + 1) / parts;
        pool.emplace_back([&fn, &out, b, e, p] { fn(b, e, out[p]); });
    }
    fn(n * (parts - 1) / parts, n, out[parts - 1]);
    for (auto& th : pool) th.join();
    return out;
}

int write_parts(const std::string& path, const char* mode, const std::vector<std::string>& parts)
{
    FILE* f = fopen(path.c_str(), mode);
    if (!f) return BCG_E_IO;
    bool ok = true;
    for (const std::string& s : parts)
        if (!s.empty() && fwrite(s.data(), 1, s.size(), f) != s.size()) ok = false;
    if (fclose(f) != 0) ok = false;
    return ok ? BCG_OK : BCG_E_IO;
}

int write_rows(const std::string& path, const std::vector<Row>& rows, int X, int threads)
{
    auto parts = in_parts(rows.size(), threads, 8, [&](size_t b, size_t e, std::string& out) {
        out.reserve((e - b) * (size_t)X * 14 + 16);
        for (size_t i = b; i < e; i++) {
            const Row& r = rows[i];
            for (int x = 0; x < X; x++)
                appendf(out, FIELD_VALUE, r.pl.p ? r.pl.p[x * r.pl.sx + (ptrdiff_t)r.z * r.pl.sz] : 0.0);
            out += r.blank ? "\n\n" : "\n";
        }
    });
    return write_parts(path, "w", parts);
}

/* mkdir -p, mode 0775 as CreateOutputFiles' mkdir calls */
int make_dirs(const std::string& dir)
{
    const mode_t mode = S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH;
    std::string p;
    for (size_t i = 0; i <= dir.size(); i++) {
        if (i == dir.size() || dir[i] == '/') {
            if (!p.empty() && mkdir(p.c_str(), mode) != 0 && errno != EEXIST) return BCG_E_IO;
        }
        if (i < dir.size()) p += dir[i];
    }
    struct stat st;
    return (stat(dir.c_str(), &st) == 0 && S_ISDIR(st.st_mode)) ? BCG_OK : BCG_E_IO;
}

int make_subdir(const std::string& dir, const char* name)
{
    std::string p = dir + "/" + name;
    if (mkdir(p.c_str(), S_IRWXU | S_IRWXG | S_IROTH | S_IXOTH) != 0 && errno != EEXIST) return BCG_E_IO;
    return BCG_OK;
}

std::string step_file(const std::string& dir, const char* name, int id)
{
    return dir + "/" + name + "/" + std::to_string(id) + ".txt";
}

int write_step(const std::string& dir, int id, int what, int append, const Step& s, int threads)
{
    int rc = make_dirs(dir);
    if (rc) return rc;
    if (what & BCG_OUT_CELLS) {
        /* CreateOutputFiles: every directory, every file opened ("w"; Cells
         * "a" when appending) */
        for (const char* name : kTree)
            if ((rc = make_subdir(dir, name))) return rc;
        for (const char* name : kTree) {
            if (!strcmp(name, "Cells")) continue;
            FILE* f = fopen(step_file(dir, name, id).c_str(), "w");
            if (!f || fclose(f) != 0) return BCG_E_IO;
        }
        auto parts = in_parts((size_t)s.n_cells, threads, 2048, [&](size_t b, size_t e, std::string& out) {
            out.reserve((e - b) * 224);
            for (size_t i = b; i < e; i++) {
                const bcg_cell& c = s.cells[i];
                const double* f = s.force + i * (size_t)s.force_stride;
                appendf(out, CELL_LINE, s.t, (int)i, c.type, c.p.x, c.p.y, c.p.z, c.q.x, c.q.y, c.q.z, c.length,
                        f[0], f[1], f[2], c.velocity.x, c.velocity.y, c.velocity.z, c.growth_rate,
                        c.dyn_fric.x, c.dyn_fric.y, c.dyn_fric.z, c.sta_fric.x, c.sta_fric.y, c.sta_fric.z,
                        c.time_p, c.time_q, c.age_p, c.age_q, c.ancestor);
            }
        });
        if ((rc = write_parts(step_file(dir, "Cells", id), append ? "a" : "w", parts))) return rc;
    }
    if (what & BCG_OUT_FIELDS) {
        const char* mine[5] = {"Restart", "Density", "Environment", "AgarField", "WallField"};
        for (const char* name : mine)
            if ((rc = make_subdir(dir, name))) return rc;
        /* SaveCells(Files.restart, new_cells, N_cells, t, dt) */
        FILE* f = fopen(step_file(dir, "Restart", id).c_str(), "w");
        if (!f) return BCG_E_IO;
        bool ok = true;
        if (s.n_restart >= 0) {
            ok = fwrite(&s.t, sizeof(double), 1, f) == 1 && fwrite(&s.dt, sizeof(double), 1, f) == 1 &&
                 (s.n_restart == 0 || fwrite(s.restart, sizeof(bcg_cell), (size_t)s.n_restart, f) == (size_t)s.n_restart);
        }
        if (fclose(f) != 0 || !ok) return BCG_E_IO;
        std::vector<Row> rows;
        for (int z = 0; z < s.Z; z++) rows.push_back({s.density, z, true});
        if ((rc = write_rows(step_file(dir, "Density", id), rows, s.X, threads))) return rc;
        rows.clear();
        for (int k = 0; k < 17; k++)
            for (int z = 0; z < s.Z; z++) rows.push_back({s.env[k], z, false});
        if ((rc = write_rows(step_file(dir, "Environment", id), rows, s.X, threads))) return rc;
        rows.clear();
        for (int l = 0; l < s.levels; l++)
            for (int m = 0; m < 4; m++)
                for (int z = 0; z < s.Za; z++) rows.push_back({s.agar[4 * l + m], z, false});
        if ((rc = write_rows(step_file(dir, "AgarField", id), rows, s.X, threads))) return rc;
        rows.clear();
        for (int l = 0; l < s.levels; l++)
            for (int m = 0; m < 4; m++) rows.push_back({s.wall[4 * l + m], 0, false});
        if ((rc = write_rows(step_file(dir, "WallField", id), rows, s.X, threads))) return rc;
    }
    return BCG_OK;
}

int hw_threads(int threads)
{
    if (threads > 0) return threads;
    unsigned h = std::thread::hardware_concurrency();
    return h ? (int)h : 1;
}

} // namespace

extern "C" int bcg_write_output(const char* dir, int output_id, int what, int append,
                                const bcg_output_data* d, int threads)
{
    if (!dir || !d || output_id < 0 || (what & ~(BCG_OUT_CELLS | BCG_OUT_FIELDS))) return BCG_E_ARG;
    Step s;
    s.t = d->t; s.dt = d->dt;
    if (what & BCG_OUT_CELLS) {
        if (d->n_cells < 0 || d->force_stride < 3 || (d->n_cells > 0 && (!d->cells || !d->cell_force))) return BCG_E_ARG;
        s.n_cells = d->n_cells; s.force_stride = d->force_stride; s.cells = d->cells; s.force = d->cell_force;
    }
    if (what & BCG_OUT_FIELDS) {
        if (d->box_x < 1 || d->box_z < 1 || d->box_z_agar < 1 || d->levels < 0) return BCG_E_ARG;
        if (d->n_restart > 0 && !d->restart_cells) return BCG_E_ARG;
        if (d->levels > 0 && (!d->agar || !d->wall)) return BCG_E_ARG;
        s.n_restart = d->n_restart; s.restart = d->restart_cells;
        s.X = d->box_x; s.Z = d->box_z; s.Za = d->box_z_agar; s.levels = d->levels;
        s.density = {d->density, d->box_z, 1};
        for (int k = 0; k < 17; k++) s.env[k] = {d->env[k], d->box_z, 1};
        for (int i = 0; i < 4 * d->levels; i++) {
            s.agar.push_back({d->agar[i], d->box_z_agar, 1});
            s.wall.push_back({d->wall[i], 1, 0});
        }
    }
    return write_step(dir, output_id, what, append, s, hw_threads(threads));
}

/* ======================================================================= */
/* asynchronous writer                                                      */
/* ======================================================================= */
namespace {
struct Slot { void* host = nullptr; size_t cap = 0; bool busy = false; };
struct Job {
    bool lineage = false;
    int id = 0;
    double t = 0, dt = 0;
    bcg_out_layout L{};
    Slot* slot = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<int> pairs;
};
} // namespace

struct bcg_writer {
    std::string dir;
    int append = 0, threads = 1, max_pending = 2;
    int device = -1;
    cudaStream_t copy = nullptr;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job*> queue;
    int in_flight = 0;      /* jobs queued or being written */
    int slot_jobs = 0;      /* of them, jobs holding a pinned slot */
    std::vector<Slot*> slots;
    int error = BCG_OK;
    bool stop = false;
    FILE* lineage = nullptr;
    std::thread th;
};

namespace {
Step step_from_snapshot(const Job& j)
{
    const bcg_out_layout& L = j.L;
    const char* base = (const char*)j.slot->host;
    Step s;
    s.t = j.t; s.dt = j.dt;
    if (L.what & BCG_OUT_CELLS) {
        s.n_cells = L.n_cells; s.force_stride = L.force_stride;
        s.cells = (const bcg_cell*)(base + L.off_cells);
        s.force = (const double*)(base + L.off_force);
    }
    if (L.what & BCG_OUT_FIELDS) {
        const size_t X = L.box_x, XZ = (size_t)L.box_x * L.box_z, XA = (size_t)L.box_x * L.box_z_agar;
        s.n_restart = L.n_restart;
        s.restart = (const bcg_cell*)(base + L.off_restart);
        s.X = L.box_x; s.Z = L.box_z; s.Za = L.box_z_agar; s.levels = L.levels;
        s.density = {(const double*)(base + L.off_density), L.box_z, 1};
        const double* env = (const double*)(base + L.off_env);
        for (int k = 0; k < 17; k++) s.env[k] = {env + k * XZ, L.box_z, 1};
        const double* ag = (const double*)(base + L.off_agar);
        const double* wl = (const double*)(base + L.off_wall);
        for (int l = 0; l < L.levels; l++) {
            /* snapshot rows are z-major; the waste member is never written */
            const ptrdiff_t sx = 1, sz = (ptrdiff_t)X;
            s.agar.push_back({ag + (3 * l + 0) * XA, sx, sz});
            s.agar.push_back({ag + (3 * l + 1) * XA, sx, sz});
            s.agar.push_back({nullptr, sx, sz});
            s.agar.push_back({ag + (3 * l + 2) * XA, sx, sz});
            for (int m = 0; m < 4; m++) s.wall.push_back({wl + (4 * l + m) * X, 1, 0});
        }
    }
    return s;
}

int run_job(bcg_writer* w, Job* j)
{
    if (j->lineage) {
        if (!w->lineage) return BCG_E_IO;
        for (size_t i = 0; i + 1 < j->pairs.size(); i += 2)
            if (fprintf(w->lineage, "%d %d\n", j->pairs[i], j->pairs[i + 1]) < 0) return BCG_E_IO;
        return BCG_OK;
    }
    cudaSetDevice(w->device);
    cudaError_t e = cudaEventSynchronize(j->done);
    if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; }
    return write_step(w->dir, j->id, j->L.what, w->append, step_from_snapshot(*j), w->threads);
}

void writer_main(bcg_writer* w)
{
    for (;;) {
        Job* j;
        {
            std::unique_lock<std::mutex> lk(w->mu);
            w->cv.wait(lk, [w] { return w->stop || !w->queue.empty(); });
            if (w->queue.empty()) return;
            j = w->queue.front();
            w->queue.pop_front();
        }
        int rc = run_job(w, j);
        if (j->done) cudaEventDestroy(j->done);
        {
            std::lock_guard<std::mutex> lk(w->mu);
            if (rc && !w->error) w->error = rc;
            if (j->slot) { j->slot->busy = false; w->slot_jobs--; }
            w->in_flight--;
        }
        w->cv.notify_all();
        delete j;
    }
}

/* a pinned slot of at least `bytes`, once fewer than max_pending steps hold one */
int acquire_slot(bcg_writer* w, size_t bytes, Slot** out)
{
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv.wait(lk, [w] { return w->slot_jobs < w->max_pending; });
    Slot* pick = nullptr;
    for (Slot* s : w->slots)
        if (!s->busy && s->cap >= bytes && (!pick || s->cap < pick->cap)) pick = s;
    if (!pick) {
        for (Slot* s : w->slots)
            if (!s->busy) { pick = s; break; }
        if (!pick) { pick = new Slot(); w->slots.push_back(pick); }
        if (pick->host) { cudaFreeHost(pick->host); pick->host = nullptr; pick->cap = 0; }
        size_t cap = std::max<size_t>(bytes, 1 << 20);
        cudaError_t e = cudaHostAlloc(&pick->host, cap, cudaHostAllocDefault);
        if (e != cudaSuccess) { pick->host = nullptr; bcg_set_cuda_error(e); return BCG_E_CUDA; }
        pick->cap = cap;
    }
    pick->busy = true;
    w->slot_jobs++;
    *out = pick;
    return BCG_OK;
}

void release_slot(bcg_writer* w, Slot* s)
{
    std::lock_guard<std::mutex> lk(w->mu);
    s->busy = false;
    w->slot_jobs--;
    w->cv.notify_all();
}

int take_error(bcg_writer* w)
{
    std::lock_guard<std::mutex> lk(w->mu);
    int rc = w->error;
    w->error = BCG_OK;
    return rc;
}

/* the writer's copy stream lives on the device of the first context */
int bind_device(bcg_writer* w, bcg_ctx* c)
{
    int dev = bcg_int_device(c);
    if (w->device >= 0) return dev == w->device ? BCG_OK : BCG_E_ARG;
    int prev = -1;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&w->copy, cudaStreamNonBlocking);
    if (prev >= 0) cudaSetDevice(prev);
    if (e != cudaSuccess) { bcg_set_cuda_error(e); return BCG_E_CUDA; }
    w->device = dev;
    return BCG_OK;
}

int submit_step(bcg_writer* w, bcg_ctx* c, int id, int what, int initial, double t, double dt, int64_t* fcw)
{
    if (!w || !c || id < 0) return BCG_E_ARG;
    int rc = bind_device(w, c);
    if (rc) return rc;
    Job* j = new Job();
    j->id = id; j->t = t; j->dt = dt;
    if ((rc = bcg_int_out_layout(c, what, initial, &j->L))) { delete j; return rc; }
    if ((rc = acquire_slot(w, j->L.bytes, &j->slot))) { delete j; return rc; }
    cudaError_t e = cudaEventCreateWithFlags(&j->done, cudaEventDisableTiming);
    if (e != cudaSuccess) { release_slot(w, j->slot); delete j; bcg_set_cuda_error(e); return BCG_E_CUDA; }
    rc = bcg_int_out_snapshot(c, &j->L, j->slot->host, w->copy, j->done, fcw);
    if (rc == BCG_E_CUDA || rc == BCG_E_ARG) {
        /* the copy may be queued: let it finish before the slot is reused */
        cudaStreamSynchronize(w->copy);
        cudaEventDestroy(j->done);
        release_slot(w, j->slot);
        delete j;
        return rc;
    }
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->queue.push_back(j);
        w->in_flight++;
    }
    w->cv.notify_all();
    if (rc) return rc;   /* a device status word (e.g. a cell out of the grid); the step is still written */
    return take_error(w);
}
} // namespace

extern "C" int bcg_writer_create(const char* dir, int append, int threads, int max_pending, bcg_writer** out)
{
    if (!dir || !out || max_pending < 1) return BCG_E_ARG;
    *out = nullptr;
    std::string d(dir);
    while (d.size() > 1 && d.back() == '/') d.pop_back();
    if (make_dirs(d) || make_subdir(d, "lineage")) return BCG_E_IO;
    bcg_writer* w = new bcg_writer();
    w->dir = d;
    w->append = append != 0;
    w->threads = hw_threads(threads);
    w->max_pending = max_pending;
    /* CreateOutputFileLineage(0, ...) opens it "w" whatever `append` is */
    w->lineage = fopen((d + "/lineage/0.txt").c_str(), "w");
    if (!w->lineage) { delete w; return BCG_E_IO; }
    w->th = std::thread(writer_main, w);
    *out = w;
    return BCG_OK;
}

extern "C" int bcg_writer_wait(bcg_writer* w)
{
    if (!w) return BCG_E_ARG;
    std::unique_lock<std::mutex> lk(w->mu);
    w->cv.wait(lk, [w] { return w->in_flight == 0; });
    if (w->lineage && fflush(w->lineage) != 0 && !w->error) w->error = BCG_E_IO;
    int rc = w->error;
    w->error = BCG_OK;
    return rc;
}

extern "C" int bcg_writer_destroy(bcg_writer* w)
{
    if (!w) return BCG_OK;
    int rc = bcg_writer_wait(w);
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->stop = true;
    }
    w->cv.notify_all();
    w->th.join();
    if (w->lineage && fclose(w->lineage) != 0 && !rc) rc = BCG_E_IO;
    for (Slot* s : w->slots) {
        if (s->host) cudaFreeHost(s->host);
        delete s;
    }
    if (w->copy) cudaStreamDestroy(w->copy);
    delete w;
    return rc;
}

extern "C" int bcg_output_initial(bcg_writer* w, bcg_ctx* ctx, double t)
{
    return submit_step(w, ctx, 0, BCG_OUT_CELLS | BCG_OUT_FIELDS, 1, t, 0.0, nullptr);
}

extern "C" int bcg_output_cells(bcg_writer* w, bcg_ctx* ctx, int output_id, double t, int64_t* fcw_calls)
{
    int64_t f = 0;
    int rc = submit_step(w, ctx, output_id, BCG_OUT_CELLS, 0, t, 0.0, &f);
    if (fcw_calls) *fcw_calls = f;
    return rc;
}

extern "C" int bcg_output_fields(bcg_writer* w, bcg_ctx* ctx, int output_id, double t, double dt)
{
    return submit_step(w, ctx, output_id, BCG_OUT_FIELDS, 0, t, dt, nullptr);
}

extern "C" int bcg_writer_lineage(bcg_writer* w, const int* pairs, int n_pairs)
{
    if (!w || n_pairs < 0 || (n_pairs > 0 && !pairs)) return BCG_E_ARG;
    if (n_pairs == 0) return take_error(w);
    Job* j = new Job();
    j->lineage = true;
    j->pairs.assign(pairs, pairs + 2 * (size_t)n_pairs);
    {
        std::lock_guard<std::mutex> lk(w->mu);
        w->queue.push_back(j);
        w->in_flight++;
    }
    w->cv.notify_all();
    return take_error(w);
}
