// Request loop over a resident database: queries served as they arrive, with
// continuous batching.
//
// The reference is a batch program: its job dispatcher hands whole queries
// to per-GPU worker threads in round robin (src/libmycu/cualn/
// JobDispatcher.cpp:1124-1133), each worker searching one query at a time
// (src/libmycu/cualn/DevCommThread.cpp:316-355). Here a server keeps one
// database chunk resident on a GPU and serves queries as they arrive:
//
//  * slots: search contexts sharing the resident chunk (cbp_share_database),
//    each with its own stream, working memory and worker thread, so that the
//    batches in flight overlap on the device;
//  * continuous batching: when a slot is free, the dispatcher takes the
//    oldest waiting query and the ones behind it, in arrival order, up to
//    max_batch, as long as the stacked queries' slab still holds the longest
//    database profile; the batch is searched in one pass over the database
//    (cbp_process_batch: one score-matrix launch over the stacked rows);
//  * admission by memory footprint: a batch is charged what its score
//    matrices, DP buffers and alignment rows take for one slab
//    (cbp_slab_bytes), the slab cut so that one batch takes at most
//    max_share of the budget; a slot's buffers only grow, so each slot is
//    charged the largest footprint it has held, and a batch is admitted
//    only while the sum over the slots stays within the budget.
//
// Everything here is host C++ over the library's own C ABI.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "cother_b200.h"

namespace {

double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
    uint64_t ticket = 0;
    size_t Lq = 0;
    std::vector<std::vector<char>> fields;   // the query's field data, copied at submission
    char* beg[CBP_NFIELDS] = {};
    char* end[CBP_NFIELDS] = {};
    double arrival = 0, start = 0, finish = 0;
    int status = 0;                          // 0 pending, 1 done, < 0 failed (-status = the code)
    std::string error;
    int slot = -1, batch = 0;
    size_t slab = 0;
    std::vector<float> recs;
    std::vector<int32_t> order;
    std::vector<char> alns;                  // 5 rows of alnlen bytes
    size_t alnlen = 0;
};
using ReqPtr = std::shared_ptr<Request>;

thread_local std::string g_server_error;

}  // namespace

struct cbp_server {
    cbp_server_config cfg{};
    cbp_options opt{};
    cbp_context* owner = nullptr;
    std::vector<cbp_context*> slots;
    size_t db_positions = 0;
    size_t longest = 0;
    size_t budget = 0;

    std::mutex mu;
    std::condition_variable cv;
    std::deque<ReqPtr> queue;
    std::map<uint64_t, ReqPtr> reqs;
    std::vector<std::vector<ReqPtr>> assigned;
    std::vector<size_t> slab_of;
    std::vector<size_t> held;       // the ledger: largest footprint each slot has held
    std::vector<char> busy;
    bool stop = false;
    uint64_t next_ticket = 1;
    std::thread dispatcher;
    std::vector<std::thread> workers;

    // bytes per slab position and per slab for `rows` stacked query rows
    void cost(size_t rows, size_t* per_pos, size_t* fixed) const
    {
        size_t b0 = 0, b1 = 0;
        cbp_slab_bytes(&opt, rows, 0, &b0);
        cbp_slab_bytes(&opt, rows, 1, &b1);
        *fixed = b0;
        *per_pos = b1 > b0 ? b1 - b0 : 1;
    }
    size_t footprint(size_t rows, size_t slab) const
    {
        size_t pp, fx;
        cost(rows, &pp, &fx);
        return fx + pp * slab;
    }
    // the largest slab whose footprint fits max_share of the budget
    size_t slab_for(size_t rows) const
    {
        size_t pp, fx;
        cost(rows, &pp, &fx);
        const double share = cfg.max_share > 0 ? cfg.max_share : 0.5;
        const double cap = (double)budget * share - (double)fx;
        const size_t s = cap > 0 ? (size_t)(cap / (double)pp) : 0;
        return std::max<size_t>(1, std::min(db_positions, s));
    }

    int choose(size_t need, size_t min_grant, size_t* grant) const
    {
        return cbp_ledger_choose(held.data(), busy.data(), held.size(), budget, need, min_grant, grant);
    }

    void dispatch()
    {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
            cv.wait(lk, [&] { return stop || !queue.empty(); });
            if (queue.empty()) return;   // stopped and drained
            // the oldest request and the ones behind it, while their stacked
            // rows still leave room for a slab of the longest profile
            const size_t whole = std::min(longest, db_positions);
            size_t rows = queue[0]->Lq, n = 1;
            const size_t maxb = (size_t)std::max(1, cfg.max_batch);
            while (n < maxb && n < queue.size() && slab_for(rows + queue[n]->Lq) >= whole) rows += queue[n++]->Lq;
            size_t slab = slab_for(rows);
            size_t need = footprint(rows, slab), grant = 0;
            const int i = choose(need, footprint(rows, whole), &grant);
            if (i < 0) {
                cv.wait(lk);
                continue;
            }
            if (grant < need) {
                size_t pp, fx;
                cost(rows, &pp, &fx);
                slab = std::min(db_positions, (grant - fx) / pp);
                need = footprint(rows, slab);
            }
            std::vector<ReqPtr> batch(queue.begin(), queue.begin() + (long)n);
            queue.erase(queue.begin(), queue.begin() + (long)n);
            busy[i] = 1;
            held[i] = std::max(held[i], need);
            slab_of[i] = slab;
            assigned[i] = std::move(batch);
            cv.notify_all();
        }
    }

    void work(size_t i)
    {
        cbp_context* ctx = slots[i];
        for (;;) {
            std::vector<ReqPtr> batch;
            size_t slab = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return !assigned[i].empty() || (stop && queue.empty()); });
                if (assigned[i].empty()) return;
                batch = assigned[i];
                slab = slab_of[i];
            }
            const double start = now_s();
            const size_t n = batch.size();
            std::vector<size_t> lens(n);
            std::vector<char* const*> begs(n), ends(n);
            for (size_t k = 0; k < n; k++) {
                lens[k] = batch[k]->Lq;
                begs[k] = batch[k]->beg;
                ends[k] = batch[k]->end;
            }
            int rc = cbp_set_max_slab_positions(ctx, slab);
            if (rc == CBP_OK) rc = cbp_process_batch(ctx, n, lens.data(), begs.data(), ends.data());
            std::string msg = rc == CBP_OK ? "" : cbp_last_error();
            for (size_t k = 0; k < n && rc == CBP_OK; k++) {
                Request& r = *batch[k];
                size_t nrec = 0, nhit = 0, len = 0;
                rc = cbp_select_query(ctx, k, nullptr);
                if (rc == CBP_OK) rc = cbp_get_hit_records(ctx, nullptr, 0, &nrec);
                if (rc == CBP_OK) {
                    r.recs.resize(nrec * CBP_REC_FLOATS);
                    rc = cbp_get_hit_records(ctx, r.recs.data(), nrec, &nrec);
                }
                if (rc == CBP_OK) rc = cbp_get_hit_list(ctx, nullptr, 0, &nhit);
                if (rc == CBP_OK) {
                    r.order.resize(nhit);
                    rc = cbp_get_hit_list(ctx, r.order.data(), nhit, &nhit);
                }
                if (rc == CBP_OK) rc = cbp_get_alignments(ctx, nullptr, 0, &len);
                if (rc == CBP_OK) {
                    r.alns.resize(5 * std::max<size_t>(len, 1));
                    r.alnlen = len;
                    rc = cbp_get_alignments(ctx, r.alns.data(), len, &len);
                }
                if (rc != CBP_OK) msg = cbp_last_error();
            }
            const double finish = now_s();
            std::lock_guard<std::mutex> lk(mu);
            for (auto& r : batch) {
                r->start = start;
                r->finish = finish;
                r->slot = (int)i;
                r->batch = (int)n;
                r->slab = slab;
                r->fields.clear();   // the query's data are no longer needed
                if (rc == CBP_OK) {
                    r->status = 1;
                } else {
                    r->status = -rc;
                    r->error = msg;
                }
            }
            assigned[i].clear();
            busy[i] = 0;
            cv.notify_all();
        }
    }
};

namespace {

template <class F>
int server_guarded(F&& f)
{
    try {
        const int rc = f();
        if (rc == CBP_OK) g_server_error.clear();
        return rc;
    } catch (const std::exception& e) {
        g_server_error = e.what();
        return CBP_ERR_ARG;
    }
}

int fail(int rc, const std::string& msg)
{
    g_server_error = msg;
    return rc;
}

ReqPtr find(cbp_server* s, uint64_t ticket)
{
    auto it = s->reqs.find(ticket);
    return it == s->reqs.end() ? nullptr : it->second;
}

}  // namespace

extern "C" {

int cbp_ledger_choose(const size_t* held, const char* busy, size_t nslots, size_t budget, size_t need,
                      size_t min_grant, size_t* grant)
{
    size_t total = 0;
    for (size_t i = 0; i < nslots; i++) total += held[i];
    int best = -1;
    size_t best_growth = 0;
    for (size_t i = 0; i < nslots; i++) {
        if (busy[i]) continue;
        const size_t growth = need > held[i] ? need - held[i] : 0;
        if (total + growth <= budget && (best < 0 || growth < best_growth)) {
            best = (int)i;
            best_growth = growth;
        }
    }
    if (best >= 0) {
        *grant = need;
        return best;
    }
    // wait while a busy slot would have room once it is done
    for (size_t i = 0; i < nslots; i++)
        if (busy[i] && total + (need > held[i] ? need - held[i] : 0) <= budget) return -1;
    // no slot will ever have room for all of it: the roomiest free slot
    int room_i = -1;
    size_t room = 0;
    for (size_t i = 0; i < nslots; i++) {
        if (busy[i]) continue;
        const size_t avail = budget - (total - held[i]);
        if (room_i < 0 || avail > room) { room = avail; room_i = (int)i; }
    }
    if (room_i >= 0 && room >= min_grant) {
        *grant = room;
        return room_i;
    }
    return -1;
}

void cbp_server_default_config(cbp_server_config* cfg)
{
    if (!cfg) return;
    cfg->device = 0;
    cfg->slots = 3;
    cfg->max_batch = 4;
    cfg->budget_bytes = 0;
    cfg->max_share = 0.5;
    cfg->db_len = 0;
    cfg->n_seqs = 0;
}

const char* cbp_server_last_error(void) { return g_server_error.c_str(); }

int cbp_server_create(const cbp_server_config* cfg, const cbp_options* opt, const float* ss_table,
                      char* const* db_beg, char* const* db_end, cbp_server** out)
{
    return server_guarded([&]() -> int {
        if (!cfg || !opt || !ss_table || !db_beg || !db_end || !out) return fail(CBP_ERR_ARG, "null argument");
        *out = nullptr;
        if (cfg->slots < 1 || cfg->slots > 64) return fail(CBP_ERR_ARG, "slots must be in [1, 64]");
        if (!(cfg->max_share > 0.0 && cfg->max_share <= 1.0)) return fail(CBP_ERR_ARG, "max_share must be in (0, 1]");
        std::unique_ptr<cbp_server> s(new cbp_server());
        s->cfg = *cfg;
        s->opt = *opt;
        int rc = cbp_create(cfg->device, opt, ss_table, (size_t)1 << 20, &s->owner);
        if (rc != CBP_OK) return fail(rc, cbp_last_error());
        rc = cbp_transfer_chunk(s->owner, db_beg, db_end, nullptr);
        if (rc != CBP_OK) {
            const std::string m = cbp_last_error();
            cbp_destroy(s->owner);
            return fail(rc, m);
        }
        constexpr int kLenField = 21;   // pps2DLen (src/libmycu/cupro/PM2DVectorFields.h)
        if (!db_beg[kLenField] || !db_end[kLenField]) return fail(CBP_ERR_ARG, "no profile lengths");
        const size_t P = (size_t)(db_end[kLenField] - db_beg[kLenField]) / sizeof(int);
        const int* lens = reinterpret_cast<const int*>(db_beg[kLenField]);
        for (size_t p = 0; p < P; p++) {
            s->db_positions += (size_t)lens[p];
            s->longest = std::max(s->longest, (size_t)lens[p]);
        }
        size_t free_b = 0, total_b = 0;
        rc = cbp_device_memory(cfg->device, &free_b, &total_b);
        s->budget = cfg->budget_bytes ? cfg->budget_bytes : (size_t)(0.7 * (double)free_b);
        const int nslots = cfg->slots;
        s->assigned.resize(nslots);
        s->slab_of.assign(nslots, 0);
        s->held.assign(nslots, 0);
        s->busy.assign(nslots, 0);
        for (int i = 0; i < nslots; i++) {
            cbp_context* c = nullptr;
            rc = cbp_create(cfg->device, opt, ss_table, s->budget, &c);
            if (rc == CBP_OK) rc = cbp_share_database(c, s->owner);
            if (rc == CBP_OK)
                rc = cbp_set_db_details(c, cfg->db_len ? cfg->db_len : s->db_positions,
                                        cfg->n_seqs ? cfg->n_seqs : P);
            if (rc != CBP_OK) {
                const std::string m = cbp_last_error();
                if (c) cbp_destroy(c);
                for (cbp_context* x : s->slots) cbp_destroy(x);
                cbp_destroy(s->owner);
                return fail(rc, m);
            }
            s->slots.push_back(c);
        }
        cbp_server* raw = s.release();
        raw->dispatcher = std::thread([raw] { raw->dispatch(); });
        for (int i = 0; i < nslots; i++) raw->workers.emplace_back([raw, i] { raw->work((size_t)i); });
        *out = raw;
        return CBP_OK;
    });
}

int cbp_server_budget(cbp_server* s, size_t* budget_bytes)
{
    if (!s || !budget_bytes) return fail(CBP_ERR_ARG, "null argument");
    *budget_bytes = s->budget;
    return CBP_OK;
}

int cbp_server_submit(cbp_server* s, size_t query_len, char* const* qbeg, char* const* qend, uint64_t* ticket)
{
    return server_guarded([&]() -> int {
        if (!s || !qbeg || !qend || !ticket) return fail(CBP_ERR_ARG, "null argument");
        auto r = std::make_shared<Request>();
        r->Lq = query_len;
        r->fields.resize(CBP_NFIELDS);
        for (int f = 0; f < CBP_NFIELDS; f++) {
            if (!qbeg[f] || !qend[f] || qend[f] < qbeg[f]) continue;
            r->fields[f].assign(qbeg[f], qend[f]);
            r->beg[f] = r->fields[f].data();
            r->end[f] = r->fields[f].data() + r->fields[f].size();
        }
        // a batch's slab must hold the longest profile
        if (s->slab_for(query_len) < std::min(s->longest, s->db_positions))
            return fail(CBP_ERR_MEMORY, "the memory budget cannot hold one slab of the longest profile for this "
                                        "query length");
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return fail(CBP_ERR_STATE, "the server is closing");
        r->ticket = s->next_ticket++;
        r->arrival = now_s();
        s->reqs[r->ticket] = r;
        s->queue.push_back(r);
        *ticket = r->ticket;
        s->cv.notify_all();
        return CBP_OK;
    });
}

int cbp_server_wait(cbp_server* s, uint64_t ticket, int timeout_ms, cbp_server_result* info)
{
    return server_guarded([&]() -> int {
        if (!s) return fail(CBP_ERR_ARG, "null server");
        std::unique_lock<std::mutex> lk(s->mu);
        ReqPtr r = find(s, ticket);
        if (!r) return fail(CBP_ERR_ARG, "unknown ticket");
        auto ready = [&] { return r->status != 0; };
        if (timeout_ms < 0) s->cv.wait(lk, ready);
        else if (!s->cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            return fail(CBP_ERR_STATE, "not done yet");
        if (info) {
            info->arrival_s = r->arrival;
            info->start_s = r->start;
            info->finish_s = r->finish;
            info->slot = r->slot;
            info->batch = r->batch;
            info->slab_positions = r->slab;
            info->nrecords = r->recs.size() / CBP_REC_FLOATS;
            info->nhits = r->order.size();
            info->alignment_length = r->alnlen;
        }
        if (r->status < 0) return fail(-r->status, r->error);
        return CBP_OK;
    });
}

int cbp_server_get(cbp_server* s, uint64_t ticket, float* records, size_t max_records, int32_t* order,
                   size_t max_hits, char* rows, size_t row_stride)
{
    return server_guarded([&]() -> int {
        if (!s) return fail(CBP_ERR_ARG, "null server");
        std::lock_guard<std::mutex> lk(s->mu);
        ReqPtr r = find(s, ticket);
        if (!r) return fail(CBP_ERR_ARG, "unknown ticket");
        if (r->status != 1) return fail(CBP_ERR_STATE, "no results for this ticket");
        const size_t nrec = r->recs.size() / CBP_REC_FLOATS;
        if (records) {
            if (max_records < nrec) return fail(CBP_ERR_ARG, "record buffer too small");
            std::memcpy(records, r->recs.data(), r->recs.size() * sizeof(float));
        }
        if (order && !r->order.empty())
            std::memcpy(order, r->order.data(), std::min(max_hits, r->order.size()) * sizeof(int32_t));
        if (rows) {
            if (row_stride < r->alnlen) return fail(CBP_ERR_ARG, "row stride smaller than the alignment rows");
            for (int k = 0; k < 5; k++)
                std::memcpy(rows + (size_t)k * row_stride, r->alns.data() + (size_t)k * r->alnlen, r->alnlen);
        }
        return CBP_OK;
    });
}

int cbp_server_release(cbp_server* s, uint64_t ticket)
{
    if (!s) return fail(CBP_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    ReqPtr r = find(s, ticket);
    if (!r) return fail(CBP_ERR_ARG, "unknown ticket");
    if (r->status == 0) return fail(CBP_ERR_STATE, "the request is not finished");
    s->reqs.erase(ticket);
    return CBP_OK;
}

int cbp_server_destroy(cbp_server* s)
{
    if (!s) return CBP_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv.notify_all();
    }
    if (s->dispatcher.joinable()) s->dispatcher.join();
    for (auto& t : s->workers)
        if (t.joinable()) t.join();
    for (cbp_context* c : s->slots) cbp_destroy(c);
    if (s->owner) cbp_destroy(s->owner);
    delete s;
    return CBP_OK;
}

}  // extern "C"
