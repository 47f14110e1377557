// A server of solve requests (no counterpart in the reference, whose callers solve one model
// at a time): resident solvers keyed by the caller's id, admitted against a device-memory
// budget with least-recently-used eviction of idle solvers, and `slots` worker threads that
// each run 1 solve at a time on its solver's own CUDA stream, so that up to `slots` requests
// are on the device together and a request that arrives while others run starts as soon as a
// slot is free.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "common.cuh"
#include "solver.cuh"

namespace femgpu {

using Clock = std::chrono::steady_clock;

struct Resident {
    std::unique_ptr<femgpu_solver> solver;
    size_t bytes = 0;
    int busy = 0;  // queued or running requests
    std::list<uint64_t>::iterator lru;
};

struct Ticket {
    uint64_t key = 0;
    const double* b = nullptr;
    double* x = nullptr;
    Clock::time_point submitted, finished;
    bool done = false;
    int status = FEMGPU_OK;
    std::string message;
    femgpu_stats stats{};
};

class Server {
   public:
    Server(int slots, size_t budget) : budget_(budget) {
        for (int k = 0; k < slots; ++k) workers_.emplace_back([this] { work(); });
    }
    ~Server() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_work_.notify_all();
        for (auto& t : workers_) t.join();
    }

    // Frees idle solvers, least recently used first, until `bytes` more fit in the budget.
    // Returns false when the busy solvers alone leave no room.
    bool reserve(size_t bytes) {
        std::unique_lock<std::mutex> g(m_);
        return make_room(bytes);
    }

    void put(uint64_t key, femgpu_solver* s) {
        std::unique_lock<std::mutex> g(m_);
        size_t bytes = s->impl.bytes();
        auto it = resident_.find(key);
        if (it != resident_.end()) {
            if (it->second.busy) throw Failure(FEMGPU_ERR_INVALID, "the key's solver is in use");
            used_ -= it->second.bytes;
            lru_.erase(it->second.lru);
            resident_.erase(it);
        }
        if (bytes > budget_)
            throw Failure(FEMGPU_ERR_TOO_LARGE, "the solver alone is larger than the budget");
        if (!make_room(bytes))
            throw Failure(FEMGPU_ERR_TOO_LARGE,
                          "the budget has no room: the resident solvers that hold it are busy");
        Resident r;
        r.solver.reset(s);
        r.bytes = bytes;
        lru_.push_front(key);
        r.lru = lru_.begin();
        used_ += bytes;
        resident_.emplace(key, std::move(r));
    }

    bool has(uint64_t key) {
        std::lock_guard<std::mutex> g(m_);
        return resident_.count(key) != 0;
    }

    uint64_t submit(uint64_t key, const double* b, double* x) {
        std::lock_guard<std::mutex> g(m_);
        auto it = resident_.find(key);
        if (it == resident_.end()) throw Failure(FEMGPU_ERR_INVALID, "no resident solver for the key");
        it->second.busy += 1;
        touch(it);
        uint64_t id = next_++;
        auto t = std::make_shared<Ticket>();
        t->key = key;
        t->b = b;
        t->x = x;
        t->submitted = Clock::now();
        tickets_[id] = t;
        queue_.push_back(id);
        cv_work_.notify_one();
        return id;
    }

    void wait(uint64_t id, femgpu_stats* st, double* latency, int* status, std::string* msg) {
        std::unique_lock<std::mutex> g(m_);
        auto it = tickets_.find(id);
        if (it == tickets_.end()) throw Failure(FEMGPU_ERR_INVALID, "unknown ticket");
        std::shared_ptr<Ticket> t = it->second;
        cv_done_.wait(g, [&] { return t->done; });
        if (st) *st = t->stats;
        if (latency)
            *latency = std::chrono::duration<double>(t->finished - t->submitted).count();
        *status = t->status;
        *msg = t->message;
        tickets_.erase(id);
    }

    size_t resident_bytes() {
        std::lock_guard<std::mutex> g(m_);
        return used_;
    }
    size_t resident_count() {
        std::lock_guard<std::mutex> g(m_);
        return resident_.size();
    }

   private:
    void touch(std::unordered_map<uint64_t, Resident>::iterator it) {
        lru_.erase(it->second.lru);
        lru_.push_front(it->first);
        it->second.lru = lru_.begin();
    }

    bool make_room(size_t bytes) {
        // Least recently used at the back of the list.
        auto k = lru_.end();
        while (used_ + bytes > budget_ && k != lru_.begin()) {
            --k;
            auto it = resident_.find(*k);
            if (it->second.busy) continue;
            used_ -= it->second.bytes;
            auto dead = k;
            ++k;
            lru_.erase(dead);
            resident_.erase(it);
        }
        return used_ + bytes <= budget_;
    }

    void work() {
        for (;;) {
            uint64_t id;
            std::shared_ptr<Ticket> t;
            femgpu_solver* s = nullptr;
            {
                std::unique_lock<std::mutex> g(m_);
                // The oldest queued request whose solver no other worker is running: each
                // solver runs 1 solve at a time (it owns 1 stream and 1 set of vectors).
                for (;;) {
                    if (stop_) return;
                    auto q = queue_.begin();
                    for (; q != queue_.end(); ++q)
                        if (!running_.count(tickets_[*q]->key)) break;
                    if (q != queue_.end()) {
                        id = *q;
                        queue_.erase(q);
                        break;
                    }
                    cv_work_.wait(g);
                }
                t = tickets_[id];
                running_.insert({t->key, 1});
                s = resident_.at(t->key).solver.get();
            }
            int status = FEMGPU_OK;
            std::string msg;
            femgpu_stats st{};
            try {
                s->impl.solve_host(t->b, t->x, nullptr, &st);
            } catch (const Failure& e) {
                status = e.code;
                msg = e.what();
            } catch (const std::exception& e) {
                status = FEMGPU_ERR_INVALID;
                msg = e.what();
            }
            {
                std::lock_guard<std::mutex> g(m_);
                running_.erase(t->key);
                auto it = resident_.find(t->key);
                if (it != resident_.end()) it->second.busy -= 1;
                t->stats = st;
                t->status = status;
                t->message = msg;
                t->finished = Clock::now();
                t->done = true;
            }
            cv_done_.notify_all();
            cv_work_.notify_all();
        }
    }

    size_t budget_ = 0, used_ = 0;
    bool stop_ = false;
    uint64_t next_ = 1;
    std::mutex m_;
    std::condition_variable cv_work_, cv_done_;
    std::unordered_map<uint64_t, Resident> resident_;
    std::list<uint64_t> lru_;
    std::deque<uint64_t> queue_;
    std::map<uint64_t, std::shared_ptr<Ticket>> tickets_;
    std::map<uint64_t, int> running_;
    std::vector<std::thread> workers_;
};

}  // namespace femgpu

struct femgpu_server {
    std::unique_ptr<femgpu::Server> impl;
};

using namespace femgpu;

template <class F>
static int server_guarded(F f) {
    try {
        f();
        return FEMGPU_OK;
    } catch (const Failure& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return FEMGPU_ERR_INVALID;
    }
}

extern "C" {

int femgpu_server_new(int slots, size_t budget_bytes, femgpu_server** out) {
    return server_guarded([&] {
        if (!out || slots < 1 || slots > 64)
            throw Failure(FEMGPU_ERR_INVALID, "slots must be 1 to 64");
        auto* s = new femgpu_server;
        s->impl = std::make_unique<Server>(slots, budget_bytes);
        *out = s;
    });
}

int femgpu_server_reserve(femgpu_server* s, size_t bytes) {
    return server_guarded([&] {
        if (!s) throw Failure(FEMGPU_ERR_INVALID, "null server");
        if (!s->impl->reserve(bytes))
            throw Failure(FEMGPU_ERR_TOO_LARGE, "the budget has no room: the resident solvers "
                                                "that hold it are busy");
    });
}

int femgpu_server_put(femgpu_server* s, uint64_t key, femgpu_solver* solver) {
    return server_guarded([&] {
        if (!s || !solver) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        s->impl->put(key, solver);
    });
}

int femgpu_server_has(femgpu_server* s, uint64_t key) { return s && s->impl->has(key) ? 1 : 0; }

int femgpu_server_submit(femgpu_server* s, uint64_t key, const double* b, double* x,
                         uint64_t* ticket) {
    return server_guarded([&] {
        if (!s || !b || !x || !ticket) throw Failure(FEMGPU_ERR_INVALID, "null argument");
        *ticket = s->impl->submit(key, b, x);
    });
}

int femgpu_server_wait(femgpu_server* s, uint64_t ticket, femgpu_stats* stats,
                       double* latency_s) {
    int status = FEMGPU_OK;
    std::string msg;
    int rc = server_guarded([&] {
        if (!s) throw Failure(FEMGPU_ERR_INVALID, "null server");
        s->impl->wait(ticket, stats, latency_s, &status, &msg);
    });
    if (rc != FEMGPU_OK) return rc;
    if (status != FEMGPU_OK) set_last_error(msg);
    return status;
}

size_t femgpu_server_resident_bytes(femgpu_server* s) { return s ? s->impl->resident_bytes() : 0; }
size_t femgpu_server_resident_count(femgpu_server* s) { return s ? s->impl->resident_count() : 0; }

void femgpu_server_free(femgpu_server* s) { delete s; }

}  // extern "C"
