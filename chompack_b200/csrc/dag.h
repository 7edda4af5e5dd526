// Helper for building task programs: tasks are created with provisional ids
// and a scheduling key, then sorted by key into the final execution order.
// Waits name either a task (wait until it has run) or a group counter (wait
// until `target` member tasks have run).  finish() checks that every wait
// points strictly backwards in the final order, which is what makes the
// persistent schedule deadlock-free.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <numeric>
#include <queue>
#include <string>
#include <array>
#include <vector>

#include "engine.h"
#include "internal.h"
#include "plan.h"

namespace chb {

struct SchedKey {
  int32_t level;   // height of the front in the supernodal tree (or sweep phase)
  int32_t step;    // step of the blocked algorithm inside the front
  int32_t rank;    // task kind inside a step
  int32_t front;
  int32_t j, i;    // tile coordinates
  bool operator<(const SchedKey& o) const {
    if (level != o.level) return level < o.level;
    if (step != o.step) return step < o.step;
    if (rank != o.rank) return rank < o.rank;
    if (front != o.front) return front < o.front;
    if (j != o.j) return j < o.j;
    return i < o.i;
  }
};

struct DagBuilder {
  struct Wait {
    int32_t id;      // task id, or group id when is_group
    int32_t target;
    bool is_group;
  };
  std::vector<Task> tasks;
  std::vector<SchedKey> keys;
  std::vector<std::vector<Wait>> waits;
  std::vector<int32_t> group_of;   // provisional group of each task (-1)
  std::vector<int32_t> group_size;
  std::vector<double> cost;        // estimated duration (microseconds); of the first part for split tasks
  // Split tasks: a task with post_cost > 0 runs its first part (cost),
  // publishes its own counter (the waiters on the task need only the first
  // part), waits for its mid waits and runs its second part (post_cost),
  // whose end is published through the task's group.  On the device the
  // waits after the first Task::cdiag ones are checked between the parts;
  // the dynamic schedule releases the task on the first ones only.
  std::vector<std::vector<int>> mid_waits;
  std::vector<double> post_cost;
  // A split task whose own counter is raised only at its end (T_TRSV): its
  // waiters follow the second part.
  std::vector<char> late_release;
  // Early signals: a task may publish a one-member group part-way through
  // (the counter index goes to its aux[3] as index + 1), so that waiters on
  // its first result do not wait for all of it.
  std::vector<int32_t> early_owner;  // per group: owning task, or -1
  std::vector<int32_t> early_of;     // per task: its early group, or -1
  std::vector<double> early_at;      // per task: estimated time of the signal after its start

  // Pooled update matrices (a scratch limit).  The builder lays the
  // workspace out as [update matrices | per-front scratch], the update
  // matrices in [0, pool_region), and declares each one as a buffer: its
  // entry tasks touch it first (every other access waits on one of them)
  // and it is dead once its exits (tasks, or groups complete) have run.
  // finish() then places the buffers of at least pool_min doubles, in
  // creation order, in a pool of at most pool_limit doubles where it can: a
  // buffer that takes memory an earlier one held makes its entry tasks wait
  // on that one's exits.  Memory is only taken from buffers whose exits
  // were all created before the taker's entry tasks, so every added wait
  // names an earlier task and the creation order stays topological.  Of the
  // windows of memory it may take, a buffer takes one whose holders are
  // done by its first use in the simulated list schedule, else (at the
  // limit) the one that makes it wait least.  finish() makes POOL_PASSES
  // placements, each from the simulated schedule of the one before, and
  // keeps the one whose simulated schedule ends first among those that
  // take at most 5 % more memory than the first placement or the limit.  Smaller buffers keep memory of their own
  // after the pool; the scratch beyond pool_region moves down behind them.
  struct PoolBuf {
    int64_t off = 0, size = 0;   // in the builder's layout (doubles)
    std::vector<int> entry;      // task ids
    std::vector<Wait> exit;      // tasks and groups
    int64_t new_off = -1;        // placement
  };
  std::vector<PoolBuf> pool;
  int64_t pool_limit = -1;       // doubles; < 0: no pooling
  int64_t pool_min = 4096;       // smaller buffers are not pooled
  int64_t pool_region = 0;
  int64_t pool_doubles = 0;      // result: the pool's size
  int64_t region_doubles = 0;    // result: pool + unpooled buffers
  int64_t pool_waits = 0;        // result: reuse waits added
  static constexpr int POOL_PASSES = 10;

  int pool_buffer(int64_t off, int64_t size) {
    pool.emplace_back();
    pool.back().off = off;
    pool.back().size = size;
    return (int)pool.size() - 1;
  }
  void pool_entry(int buf, int task) {
    if (buf >= 0 && task >= 0) pool[buf].entry.push_back(task);
  }
  void pool_exit_task(int buf, int task) {
    if (buf >= 0 && task >= 0) pool[buf].exit.push_back({task, 1, false});
  }
  void pool_exit_group(int buf, int group) {
    if (buf >= 0 && group >= 0) pool[buf].exit.push_back({group, -1, true});
  }

  int new_group() {
    group_size.push_back(0);
    early_owner.push_back(-1);
    return (int)group_size.size() - 1;
  }

  int add(const Task& t, const SchedKey& key, int group = -1, double est_us = -1.0) {
    tasks.push_back(t);
    keys.push_back(key);
    cost.push_back(est_us >= 0 ? est_us : estimate(t));
    waits.emplace_back();
    mid_waits.emplace_back();
    post_cost.push_back(0.0);
    late_release.push_back(0);
    group_of.push_back(group);
    early_of.push_back(-1);
    early_at.push_back(0.0);
    if (group >= 0) group_size[group]++;
    return (int)tasks.size() - 1;
  }

  // The early-signal group of `task` (created on first use).
  int early_signal(int task, double after_us) {
    if (early_of[task] >= 0) return early_of[task];
    const int g = new_group();
    group_size[g] = 1;
    early_owner[g] = task;
    early_of[task] = g;
    early_at[task] = after_us;
    return g;
  }

  void wait_task(int task, int dep) {
    if (dep >= 0) waits[task].push_back({dep, 1, false});
  }
  // A wait checked between the two parts of a split task (post_us: the
  // estimated duration of its second part).
  void wait_mid(int task, int dep) {
    if (dep >= 0) mid_waits[task].push_back(dep);
  }
  void split_task(int task, double post_us, bool own_at_end = false) {
    post_cost[task] = post_us;
    late_release[task] = own_at_end ? 1 : 0;
  }
  // Wait for all members of a group (the group must be complete when the
  // program is finished).
  void wait_group(int task, int group) {
    if (group >= 0) waits[task].push_back({group, -1, true});
  }

  // Incoming chunks (whole supernodes) that a task reads or writes: those
  // holding the start of each operand on the values (base B_X).
  static void in_chunks(const Task& t, const IoSpec& io, std::vector<int>& out) {
    out.clear();
    if (t.op == T_NOP || t.op == T_SIGNAL || t.op == T_ARRIVAL) return;
    auto add_off = [&](int64_t off) {
      const int j = (int)(std::upper_bound(io.in_off.begin(), io.in_off.end(), off) - io.in_off.begin()) - 1;
      if (j >= 0 && j + 1 < (int)io.in_off.size() && std::find(out.begin(), out.end(), j) == out.end())
        out.push_back(j);
    };
    if (t.op == T_SUBTREE || t.op == T_PSUBTREE) {  // every chunk of [a.off, b.off)
      const auto& v = io.in_off;
      int j = (int)(std::upper_bound(v.begin(), v.end(), t.a.off) - v.begin()) - 1;
      for (j = std::max(j, 0); j + 1 < (int)v.size() && v[j] < t.b.off; j++) out.push_back(j);
      return;
    }
    for (const Operand* o : {&t.a, &t.b, &t.c})
      if (o->base == B_X && o->ld > 0) add_off(o->off);
    if (t.op == T_MROW && t.aux[0] == B_X) add_off((int64_t)(uint32_t)t.aux[2] | ((int64_t)t.aux[3] << 32));
  }

  // Outgoing chunks that a task's writes to the values overlap.  A written
  // tile of at most e rows and columns (e = max(m, n)) spans
  // [off, off + (e-1)*ld + e); a plain copy its m x n strip; a small front
  // its block; an extend-add writes the front's columns [aux[1], aux[2]).
  static void out_chunks(const Task& t, const IoSpec& io, std::vector<int>& out) {
    out.clear();
    auto add_range = [&](int64_t lo, int64_t hi) {
      const auto& v = io.out_off;
      int j = (int)(std::upper_bound(v.begin(), v.end(), lo) - v.begin()) - 1;
      for (j = std::max(j, 0); j + 1 < (int)v.size() && v[j] < hi; j++)
        if (std::find(out.begin(), out.end(), j) == out.end()) out.push_back(j);
    };
    const int64_t e = std::max(std::max(t.m, t.n), 1);
    auto tile = [&](const Operand& o) {
      if (o.base == B_X && o.ld > 0) add_range(o.off, o.off + (e - 1) * o.ld + e);
    };
    switch (t.op) {
      case T_NOP: case T_SIGNAL: case T_ARRIVAL: case T_EXTRACT: break;  // an extract writes the workspace
      case T_SUBTREE:  // the blocks of its ranges, within [a.off, b.off)
      case T_PSUBTREE:
        add_range(t.a.off, t.b.off);
        break;
      case T_FRONT:  // the front's whole nj x nn block (its update matrices are workspace)
      case T_PFRONT:
        if (t.a.base == B_X && t.a.ld > 0) add_range(t.a.off, t.a.off + (int64_t)t.m * t.n);
        break;
      case T_COPY:
        // a plain copy writes its m x n strip; the (anti-)transposing ones a square
        if ((t.aux[0] & 24) == 0 && t.c.base == B_X && t.c.ld > 0)
          add_range(t.c.off, t.c.off + (int64_t)(std::max(t.n, 1) - 1) * t.c.ld + std::max(t.m, 1));
        else
          tile(t.c);
        break;
      case T_GEMM: case T_MROW: case T_SUM: tile(t.c); break;
      case T_LA: tile(t.a); tile(t.c); break;
      case T_POTRF: tile(t.a); if (t.aux[1]) tile(t.c); break;
      case T_ASM:
        if (t.a.base == B_X && t.a.ld > 0) add_range(t.a.off + (int64_t)t.aux[1] * t.a.ld, t.a.off + (int64_t)t.aux[2] * t.a.ld);
        tile(t.c);
        break;
      default: tile(t.a); tile(t.b); tile(t.c); break;
    }
  }

  // Streaming of the values (see IoSpec): per incoming chunk a T_ARRIVAL
  // task (it waits for the host's copy, its estimated duration is the
  // chunk's arrival time) that every task touching the chunk waits on; per
  // outgoing chunk a fan-in of T_NOP tasks (at most 64 waits each, so that
  // no single task walks a long wait list) under one T_SIGNAL.  Arrival
  // tasks are created after the sweep's tasks, which breaks the creation
  // order's topology; finish() ranks and orders them first.
  std::vector<int> arrival_of_chunk;  // T_ARRIVAL task of each incoming chunk

  void apply_io(const IoSpec& io, std::vector<int>& signal_of_chunk) {
    signal_of_chunk.clear();
    arrival_of_chunk.clear();
    if (!io.in && !io.out) return;
    const int nin = io.in ? (int)io.in_off.size() - 1 : 0;
    const int nch = io.out ? (int)io.out_off.size() - 1 : 0;
    const int nt0 = (int)tasks.size();
    std::vector<int> arr(nin, -1);
    if (io.in)
      for (int j = 0; j < nin; j++) {
        Task a;
        std::memset(&a, 0, sizeof(a));
        a.op = T_ARRIVAL;
        a.aux[0] = j;
        arr[j] = add(a, SchedKey{-1, 0, 0, 0, j, 0}, -1, io.arrive_us[j]);
      }
    arrival_of_chunk = arr;
    std::vector<std::vector<int>> touch(nch);
    std::vector<int> ch;
    for (int t = 0; t < nt0; t++) {
      if (io.in) {
        in_chunks(tasks[t], io, ch);
        for (int j : ch) wait_task(t, arr[j]);
      }
      if (io.out) {
        out_chunks(tasks[t], io, ch);
        for (int j : ch) touch[j].push_back(t);
      }
    }
    if (!io.out) return;
    signal_of_chunk.assign(nch, -1);
    for (int j = 0; j < nch; j++) {
      std::vector<int> level = touch[j];
      SchedKey key{1 << 30, 0, 0, 0, j, 0};
      while (level.size() > 64) {
        std::vector<int> up;
        for (size_t i = 0; i < level.size(); i += 64) {
          Task n;
          std::memset(&n, 0, sizeof(n));
          n.op = T_NOP;
          const int id = add(n, key, -1, 0.5);
          for (size_t u = i; u < std::min(level.size(), i + 64); u++) wait_task(id, level[u]);
          up.push_back(id);
        }
        level.swap(up);
      }
      Task sg;
      std::memset(&sg, 0, sizeof(sg));
      sg.op = T_SIGNAL;
      sg.aux[0] = j;
      const int id = add(sg, key, -1, 0.5);
      for (int u : level) wait_task(id, u);
      signal_of_chunk[j] = id;
    }
  }

  // Rough duration model of a task on one CTA (microseconds); only the
  // relative sizes matter for the priority order.
  static double estimate(const Task& t) {
    // fitted to per-task traces of the 40^3 sweeps on B200
    const double mnk = (double)t.m * t.n * t.k / (64.0 * 64.0 * 64.0);
    switch (t.op) {
      case T_GEMM: return 3.0 + 6.0 * mnk;
      case T_MROW: return 11.0 + 6.0 * mnk;
      case T_LA: return 15.0;
      case T_POTRF: {
        // invert-only : factor + inverse, for the 16-column blocks that meet
        // the tile (a full tile has four)
        const double nb = (double)((t.m + 15) / 16);
        return (t.aux[2] ? 11.0 : 27.0) * (0.25 + 0.1875 * nb);
      }
      case T_SUM: return 3.0 + 0.5 * t.aux[0];
      case T_TRSV: return 1.0;  // the operand copies issued before its mid waits
      case T_COPY: return 3.5;
      default: return 6.0;
    }
  }

  // Placement of the pooled buffers (see PoolBuf) from a simulated schedule
  // (start and end time of every task), with the reuse waits it needs.
  int place_pool(const std::vector<double>& start, const std::vector<double>& endt,
                 const std::vector<std::vector<int>>& members) {
    const int nb = (int)pool.size();
    pool_waits = 0;
    for (PoolBuf& p : pool) p.new_off = -1;
    std::vector<int> emin(nb, INT32_MAX), xmax(nb, -1);
    std::vector<double> ta(nb, 0.0), tf(nb, 0.0);
    std::vector<int> cand;
    for (int b = 0; b < nb; b++) {
      PoolBuf& p = pool[b];
      if (p.off < 0 || p.size < 0 || p.off + p.size > pool_region)
        return set_error(-24, "pooled buffer %d outside the update-matrix region", b);
      double t0 = 1e300;
      for (int e : p.entry) {
        emin[b] = std::min(emin[b], e);
        t0 = std::min(t0, start[e]);
      }
      for (const Wait& w : p.exit) {
        if (w.is_group) {
          for (int u : members[w.id]) {
            xmax[b] = std::max(xmax[b], u);
            tf[b] = std::max(tf[b], endt[u]);
          }
        } else {
          xmax[b] = std::max(xmax[b], w.id);
          tf[b] = std::max(tf[b], endt[w.id]);
        }
      }
      ta[b] = t0;
      if (p.size >= pool_min && !p.entry.empty() && xmax[b] >= 0) cand.push_back(b);
    }
    // in creation order, in which a buffer's memory becomes legal to take:
    // the order of the reference's postorder stack for a bottom-up sweep
    std::stable_sort(cand.begin(), cand.end(), [&](int x, int y) { return emin[x] < emin[y]; });
    // the pool as contiguous blocks, each last held by `owner` (-1: never)
    struct Blk {
      int64_t off, size;
      int owner;
    };
    std::vector<Blk> blks;
    int64_t psize = 0;
    for (int b : cand) {
      const int64_t s = pool[b].size;
      // best window of consecutive blocks from i: no delay, then least
      // delay, then least growth of the pool, then least waste
      int bi = -1, bj = -1;
      double bdelay = 0.0;
      int64_t bext = 0, bwaste = 0;
      bool have = false;
      for (int i = 0; i <= (int)blks.size(); i++) {
        int64_t acc = 0;
        double ready = -1e300;
        bool ok = true;
        int j = i;
        for (; j < (int)blks.size() && acc < s; j++) {
          const int o = blks[j].owner;
          if (o >= 0 && xmax[o] >= emin[b]) {
            ok = false;
            break;
          }
          if (o >= 0) ready = std::max(ready, tf[o]);
          acc += blks[j].size;
        }
        if (!ok) continue;
        const int64_t ext = acc < s ? s - acc : 0;
        if (ext > 0 && psize + ext > pool_limit && (have || i < (int)blks.size())) continue;
        const double delay = std::max(0.0, ready - ta[b]);
        const int64_t waste = acc > s ? acc - s : 0;
        const bool better = !have || ((delay > 0.0) != (bdelay > 0.0) ? delay <= 0.0
                                      : delay != bdelay ? delay < bdelay
                                      : ext != bext ? ext < bext : waste < bwaste);
        if (better) {
          have = true;
          bi = i;
          bj = j;
          bdelay = delay;
          bext = ext;
          bwaste = waste;
        }
        if (i == (int)blks.size()) break;
      }
      // waits on every earlier holder of the window, once per holder
      std::vector<int> owners;
      for (int j = bi; j < bj; j++)
        if (blks[j].owner >= 0 && std::find(owners.begin(), owners.end(), blks[j].owner) == owners.end())
          owners.push_back(blks[j].owner);
      for (int o : owners)
        for (int e : pool[b].entry)
          for (const Wait& w : pool[o].exit) {
            waits[e].push_back(w);
            pool_waits++;
          }
      const int64_t off = bi < (int)blks.size() ? blks[bi].off : psize;
      int64_t acc = 0;
      for (int j = bi; j < bj; j++) acc += blks[j].size;
      Blk nb_ = {off, s, b};
      std::vector<Blk> repl(1, nb_);
      if (acc > s) repl.push_back({off + s, acc - s, blks[bj - 1].owner});
      blks.erase(blks.begin() + bi, blks.begin() + bj);
      blks.insert(blks.begin() + bi, repl.begin(), repl.end());
      if (acc < s) psize += s - acc;
      pool[b].new_off = off;
    }
    // unpooled buffers after the pool, in their old order
    int64_t next = psize;
    std::vector<int> by_off(nb);
    std::iota(by_off.begin(), by_off.end(), 0);
    std::stable_sort(by_off.begin(), by_off.end(), [&](int x, int y) { return pool[x].off < pool[y].off; });
    for (int b : by_off)
      if (pool[b].new_off < 0) {
        pool[b].new_off = next;
        next += pool[b].size;
      }
    pool_doubles = psize;
    region_doubles = next;
    return 0;
  }

  // The workspace offsets of every task rewritten to the placed layout.
  int remap_pool(Program& prog) {
    const int nb = (int)pool.size();
    std::vector<int> by_off(nb);
    std::iota(by_off.begin(), by_off.end(), 0);
    std::stable_sort(by_off.begin(), by_off.end(), [&](int x, int y) { return pool[x].off < pool[y].off; });
    // rewrite the workspace offsets: inside a buffer -> its placement;
    // past the region -> moved down; elsewhere in the region (operands of
    // empty extents) -> 0
    std::vector<int64_t> offs(nb);
    for (int i = 0; i < nb; i++) offs[i] = pool[by_off[i]].off;
    auto remap = [this, offs, by_off](int64_t o) -> int64_t {
      if (o >= pool_region) return o - pool_region + region_doubles;
      for (int i = (int)(std::upper_bound(offs.begin(), offs.end(), o) - offs.begin()) - 1; i >= 0; i--) {
        const PoolBuf& p = pool[by_off[i]];  // p.off <= o
        if (o < p.off + p.size) return p.new_off + (o - p.off);
        if (p.size > 0) break;  // buffers do not overlap: o lies in none
      }
      return 0;
    };
    for (Task& t : tasks) {
      if (t.off2 != 0) return set_error(-24, "pooled update matrices: task with an update-region offset");
      for (Operand* o : {&t.a, &t.b, &t.c})
        if (o->base == B_WS) o->off = remap(o->off);
      if (t.op == T_MROW && t.aux[0] == B_WS) {
        const int64_t m = remap((int64_t)(uint32_t)t.aux[2] | ((int64_t)t.aux[3] << 32));
        t.aux[2] = (int32_t)(uint32_t)(m & 0xffffffffLL);
        t.aux[3] = (int32_t)(m >> 32);
      }
    }
    pool_remap = remap;
    prog.ws_doubles -= pool_region - region_doubles;
    return 0;
  }
  std::function<int64_t(int64_t)> pool_remap;

  // Sort into execution order and emit the device program.
  //
  // The order is the start order of a simulated list schedule on `slots`
  // virtual CTAs: whenever a slot is free it starts the ready task with the
  // largest upward rank (longest estimated path from the task to the end of
  // the sweep).  A task starts only after everything it waits on has
  // finished, so ordering by simulated start time is topological, and the
  // device's CTAs, which claim tasks in list order, follow a schedule that
  // keeps the critical path moving while ready work fills the machine.
  int finish(Program& prog, int slots = 296) {
    std::vector<int> signal_of_chunk;
    apply_io(prog.io, signal_of_chunk);
    const int nt = (int)tasks.size();
    const int ng = (int)group_size.size();
    std::vector<std::vector<int>> members(ng);
    for (int t = 0; t < nt; t++)
      if (group_of[t] >= 0) members[group_of[t]].push_back(t);
    std::vector<double> rank(nt, 0.0), start(nt, 0.0), extra(nt, 0.0), endt(nt, 0.0);
    auto compute_rank = [&]() {
      std::fill(rank.begin(), rank.end(), 0.0);
      // creation order is topological (every wait names an earlier task)
      for (int t = nt - 1; t >= 0; t--) {
        rank[t] += cost[t] + post_cost[t] + extra[t];
        for (int d : mid_waits[t])
          if (d < t) rank[d] = std::max(rank[d], rank[t] - cost[t]);
        for (const Wait& wt : waits[t]) {
          if (wt.is_group) {
            const int o = early_owner[wt.id];
            if (o >= 0 && o < t) rank[o] = std::max(rank[o], rank[t] + early_at[o] - cost[o] - post_cost[o]);
            for (int u : members[wt.id])
              if (u < t) rank[u] = std::max(rank[u], rank[t]);
          } else if (wt.id < t) {
            // a split task's own waiters follow its first part only (its
            // end, for a task that raises its counter at the end)
            rank[wt.id] = std::max(rank[wt.id], rank[t] - (late_release[wt.id] ? 0.0 : post_cost[wt.id]));
          }
        }
      }
    };
    // waiters of each task / group, and unmet wait counts
    std::vector<std::vector<int>> task_waiters(nt), group_waiters(ng);
    std::vector<int> unmet0(nt, 0);
    auto find_waiters = [&]() {
      for (auto& v : task_waiters) v.clear();
      for (auto& v : group_waiters) v.clear();
      std::fill(unmet0.begin(), unmet0.end(), 0);
      for (int t = 0; t < nt; t++) {
        for (const Wait& wt : waits[t]) {
          if (wt.is_group) {
            if (group_size[wt.id] == 0) continue;
            group_waiters[wt.id].push_back(t);
          } else {
            task_waiters[wt.id].push_back(t);
          }
          unmet0[t]++;
        }
      }
    };
    find_waiters();
    std::vector<std::vector<int>> mid_waiters(nt);
    std::vector<int> mid_unmet0(nt, 0);
    for (int t = 0; t < nt; t++)
      for (int d : mid_waits[t]) {
        mid_waiters[d].push_back(t);
        mid_unmet0[t]++;
      }
    auto simulate = [&]() -> int {
      std::vector<int> unmet = unmet0, mid_unmet = mid_unmet0;
      std::vector<char> first_done(nt, 0);
      std::vector<int> group_left(group_size.begin(), group_size.end());
      {
        auto by_rank = [&](int a, int b) { return rank[a] < rank[b] || (rank[a] == rank[b] && b < a); };
        std::priority_queue<int, std::vector<int>, decltype(by_rank)> ready(by_rank);
        typedef std::pair<double, int> Ev;
        std::priority_queue<Ev, std::vector<Ev>, std::greater<Ev>> running;
        for (int t = 0; t < nt; t++)
          if (unmet[t] == 0) ready.push(t);
        int free_slots = std::max(slots, 1);
        double now = 0.0;
        int done = 0;
        auto release = [&](int w) {
          if (--unmet[w] == 0) ready.push(w);
        };
        // second part of a split task: its end, and its early signal (its
        // estimate counts from the task's start as if it never waited)
        auto second_part = [&](int t) {
          running.push({now + std::max(post_cost[t], 1e-3), t});
          if (early_of[t] >= 0) running.push({now + std::max(early_at[t] - cost[t], 0.0), -1 - early_of[t]});
        };
        while (done < nt) {
          while (free_slots > 0 && !ready.empty()) {
            int t = ready.top();
            ready.pop();
            start[t] = now;
            if (post_cost[t] > 0.0) {
              running.push({now + std::max(cost[t], 1e-3), -1 - ng - t});
            } else {
              running.push({now + std::max(cost[t], 1e-3), t});
              if (early_of[t] >= 0) running.push({now + std::min(early_at[t], cost[t]), -1 - early_of[t]});
            }
            free_slots--;
          }
          if (running.empty()) return set_error(-23, "task graph: unsatisfiable waits");
          Ev e = running.top();
          running.pop();
          now = e.first;
          if (e.second < -ng) {  // first part of a split task done: its own waiters go
            const int t = -1 - ng - e.second;
            first_done[t] = 1;
            if (!late_release[t])
              for (int w : task_waiters[t]) release(w);
            if (mid_unmet[t] == 0) second_part(t);
            continue;
          }
          if (e.second < 0) {  // an early signal: release its waiters, no slot freed
            for (int w : group_waiters[-1 - e.second]) release(w);
            continue;
          }
          free_slots++;
          done++;
          const int t = e.second;
          endt[t] = now;
          if (post_cost[t] <= 0.0 || late_release[t])
            for (int w : task_waiters[t]) release(w);
          for (int w : mid_waiters[t])
            if (--mid_unmet[w] == 0 && first_done[w]) second_part(w);
          if (group_of[t] >= 0 && --group_left[group_of[t]] == 0)
            for (int w : group_waiters[group_of[t]]) release(w);
        }
      }
      return 0;
    };
    // Output signals: a signal's rank includes the copy time of its chunk
    // and of every chunk signalled after it (at ~50 GB/s), so that the tasks
    // that complete a chunk rank as if the copies were the rest of the sweep
    // (otherwise nothing waits on them and the schedule leaves them last).
    compute_rank();
    if (simulate() != 0) return -23;
    if (pool_limit >= 0 && !pool.empty()) {
      // a few placements, each from the simulated schedule of the one
      // before (the first from the schedule without reuse waits); the one
      // whose simulated schedule ends first is kept
      const std::vector<std::vector<Wait>> plain = waits;
      std::vector<std::vector<Wait>> best_waits;
      std::vector<int64_t> best_off(pool.size());
      int64_t best_psize = 0, best_region = 0, best_nw = 0;
      double best_span = 0.0;
      int64_t first_region = 0;
      for (int pass = 0; pass < POOL_PASSES; pass++) {
        if (pass > 0) waits = plain;
        const int rc = place_pool(start, endt, members);
        if (rc) return rc;
        find_waiters();
        compute_rank();
        if (simulate() != 0) return -23;
        // (a pass may take at most 5 % more memory than the first one, or
        // than the limit)
        const double span = *std::max_element(endt.begin(), endt.end());
        if (pass == 0) first_region = region_doubles;
        const bool fits = (double)region_doubles <= 1.05 * (double)std::max(first_region, pool_limit);
        if (pass == 0 || (span < best_span && fits)) {
          best_span = span;
          best_waits = waits;
          for (size_t b = 0; b < pool.size(); b++) best_off[b] = pool[b].new_off;
          best_psize = pool_doubles;
          best_region = region_doubles;
          best_nw = pool_waits;
        }
      }
      waits.swap(best_waits);
      for (size_t b = 0; b < pool.size(); b++) pool[b].new_off = best_off[b];
      pool_doubles = best_psize;
      region_doubles = best_region;
      pool_waits = best_nw;
      const int rc = remap_pool(prog);
      if (rc) return rc;
      find_waiters();
      compute_rank();
      if (simulate() != 0) return -23;
    }
    if (!arrival_of_chunk.empty()) {
      // Incoming copies in earliest-deadline order: chunk j is due at the
      // latest start (critical path minus upward rank) of the first task
      // that touches it; each arrival task's duration becomes the time its
      // chunk arrives in that order (~50 GB/s).
      const int nin = (int)arrival_of_chunk.size();
      double tend = 0.0;
      for (int t = 0; t < nt; t++) tend = std::max(tend, rank[t]);
      std::vector<double> due(nin, tend);
      std::vector<int> chunk_of_arrival(nt, -1);
      for (int j = 0; j < nin; j++) chunk_of_arrival[arrival_of_chunk[j]] = j;
      for (int t = 0; t < nt; t++)
        for (const Wait& wt : waits[t])
          if (!wt.is_group && chunk_of_arrival[wt.id] >= 0) {
            const int j = chunk_of_arrival[wt.id];
            due[j] = std::min(due[j], tend - rank[t]);
          }
      std::vector<int>& ord = prog.io.in_order;
      ord.resize(nin);
      std::iota(ord.begin(), ord.end(), 0);
      std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return due[x] < due[y]; });
      double at = 0.0;
      for (int j : ord) {
        at += (prog.io.in_off[j + 1] - prog.io.in_off[j]) * 8.0 / 5e4;
        cost[arrival_of_chunk[j]] = at;
      }
      compute_rank();
      if (simulate() != 0) return -23;
    }
    if (!signal_of_chunk.empty()) {
      const int nch = (int)signal_of_chunk.size();
      std::vector<int> ch(nch);
      std::iota(ch.begin(), ch.end(), 0);
      std::sort(ch.begin(), ch.end(),
                [&](int x, int y) { return start[signal_of_chunk[x]] < start[signal_of_chunk[y]]; });
      double tail = 0.0;
      for (int i = nch - 1; i >= 0; i--) {
        const int j = ch[i];
        tail += (prog.io.out_off[j + 1] - prog.io.out_off[j]) * 8.0 / 5e4;
        extra[signal_of_chunk[j]] = tail;
      }
      compute_rank();
      if (simulate() != 0) return -23;
    }
    prog.sim_span_us = nt > 0 ? *std::max_element(endt.begin(), endt.end()) : 0.0;
    std::vector<int> order(nt);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      if (start[a] != start[b]) return start[a] < start[b];
      if (rank[a] != rank[b]) return rank[a] > rank[b];
      return keys[a] < keys[b];
    });
    std::vector<int> pos(nt);
    for (int i = 0; i < nt; i++) pos[order[i]] = i;
    // latest member position of each group
    std::vector<int> gmax(group_size.size(), -1);
    for (int t = 0; t < nt; t++)
      if (group_of[t] >= 0) gmax[group_of[t]] = std::max(gmax[group_of[t]], pos[t]);
    for (size_t g = 0; g < group_size.size(); g++)
      if (early_owner[g] >= 0) gmax[g] = pos[early_owner[g]];
    prog.tasks.resize(nt);
    prog.waits.clear();
    for (int i = 0; i < nt; i++) {
      const int t = order[i];
      Task tk = tasks[t];
      tk.wait_off = (int32_t)prog.waits.size();
      // de-duplicate waits
      std::vector<int2> w;
      for (const Wait& wt : waits[t]) {
        int2 e;
        if (wt.is_group) {
          if (group_size[wt.id] == 0) continue;
          if (gmax[wt.id] >= i)
            return set_error(-20, "task graph: group wait does not point backwards (task %d)", i);
          e.x = nt + wt.id;
          e.y = group_size[wt.id];
        } else {
          if (pos[wt.id] >= i)
            return set_error(-21, "task graph: wait does not point backwards (task %d -> %d)", i, pos[wt.id]);
          e.x = pos[wt.id];
          e.y = 1;
        }
        bool dup = false;
        for (const int2& x : w)
          if (x.x == e.x) { dup = true; break; }
        if (!dup) w.push_back(e);
      }
      if (!mid_waits[t].empty() || post_cost[t] > 0.0) {
        // Mid waits may point forwards in the list: every task that needs
        // this one starts (in the simulated schedule that gives the list
        // order) after its second part, hence after each mid wait, so the
        // list order stays deadlock-free for tasks claimed in order.
        tk.cdiag = (int32_t)w.size();
        for (int d : mid_waits[t]) {
          int2 e;
          e.x = pos[d];
          e.y = 1;
          bool dup = false;
          for (const int2& x : w)
            if (x.x == e.x) { dup = true; break; }
          if (!dup) w.push_back(e);
        }
      }
      if (w.size() > 65535) return set_error(-22, "task graph: too many waits");
      tk.nwait = (uint16_t)w.size();
      tk.group = group_of[t] >= 0 ? nt + group_of[t] : -1;
      if (early_of[t] >= 0) tk.aux[3] = nt + early_of[t] + 1;  // early counter, index + 1
      prog.waits.insert(prog.waits.end(), w.begin(), w.end());
      prog.tasks[i] = tk;
    }
    prog.ncounters = (int64_t)nt + (int64_t)ng;
    prog.out_order.clear();
    if (!signal_of_chunk.empty()) {
      std::vector<int> ch(signal_of_chunk.size());
      std::iota(ch.begin(), ch.end(), 0);
      std::sort(ch.begin(), ch.end(), [&](int x, int y) { return pos[signal_of_chunk[x]] < pos[signal_of_chunk[y]]; });
      prog.out_order = ch;
    }
    // dynamic scheduling data: waits per task, waiters per counter, the
    // value at which each counter is complete, the initially ready tasks
    const int64_t nc = prog.ncounters;
    prog.npend.assign(nt, 0);
    prog.succ_off.assign(nc + 1, 0);
    prog.ctarget.assign(nc, 1);
    for (size_t g = 0; g < group_size.size(); g++) prog.ctarget[nt + g] = std::max(group_size[g], 1);
    // (a T_TRSV task is released on all its waits: under the dynamic
    // schedule it never spins on its mid waits, so ready steps cannot hold
    // every CTA while their predecessors wait for one)
    auto npre = [](const Task& tk) { return (tk.op == T_POTRF && tk.k > 0) ? (int)tk.cdiag : (int)tk.nwait; };
    for (int i = 0; i < nt; i++) {
      const Task& tk = prog.tasks[i];
      prog.npend[i] = npre(tk);
      for (int w = 0; w < npre(tk); w++) prog.succ_off[prog.waits[tk.wait_off + w].x + 1]++;
    }
    for (int64_t c = 0; c < nc; c++) prog.succ_off[c + 1] += prog.succ_off[c];
    prog.succ.assign(prog.succ_off[nc], 0);
    {
      std::vector<int> fill(prog.succ_off.begin(), prog.succ_off.end() - 1);
      for (int i = 0; i < nt; i++) {
        const Task& tk = prog.tasks[i];
        for (int w = 0; w < npre(tk); w++) prog.succ[fill[prog.waits[tk.wait_off + w].x]++] = i;
      }
    }
    const int nwords = (nt + 63) / 64, nsumm = (nwords + 63) / 64;
    prog.ready0.assign(nwords, 0ull);
    prog.summ0.assign(nsumm, 0ull);
    for (int i = 0; i < nt; i++)
      if (prog.npend[i] == 0) {
        prog.ready0[i >> 6] |= 1ull << (i & 63);
        prog.summ0[i >> 12] |= 1ull << ((i >> 6) & 63);
      }
    return 0;
  }
};

// Program-build options: the plan's value (chb_plan_set_option) when set,
// else the environment variable, else the built-in default.
inline int64_t plan_option(const chb_plan& P, int opt, const char* env, int64_t dflt) {
  if (opt >= 0 && opt < CHB_OPT_COUNT && P.opt[opt] >= 0) return P.opt[opt];
  const char* e = std::getenv(env);
  return e ? (int64_t)std::atoll(e) : dflt;
}

// Largest K of one partial product of projected_inverse's long-K tiles
// (CHB_OPT_PINV_KSPLIT / CHB_PINV_KSPLIT, rounded down to a multiple of TILE,
// at least 2 TILE; default 512: at 40^3 the sweep is bound by the CTAs'
// total work, and 384 / 512 / 768 / 1024 / 1536 gave 6.01 / 5.64 / 5.74 /
// 5.72 / 6.09 ms).
inline int pinv_ksplit(const chb_plan& P) {
  const int v = (int)(plan_option(P, CHB_OPT_PINV_KSPLIT, "CHB_PINV_KSPLIT", 512) / TILE) * TILE;
  return v < 2 * TILE ? 2 * TILE : v;
}

// Largest K of one partial product of cholesky's Schur-complement tiles
// U_k -= S_k S_k^T (CHB_OPT_CHOL_KSPLIT / CHB_CHOL_KSPLIT, rounded down to a
// multiple of TILE; 0, the default, leaves them whole).
inline int chol_ksplit(const chb_plan& P) {
  const int v = (int)(plan_option(P, CHB_OPT_CHOL_KSPLIT, "CHB_CHOL_KSPLIT", 0) / TILE) * TILE;
  return v <= 0 ? 0 : (v < 2 * TILE ? 2 * TILE : v);
}

// Largest front order (nj) that a sweep runs as one shared-memory task
// (cholesky, projected_inverse): TILE, or CHB_OPT_SMALL_FRONT_NJ /
// CHB_SMALL_FRONT_NJ when set (0 turns the small-front tasks off).
inline int small_front_nj(const chb_plan& P) {
  const int64_t v = plan_option(P, CHB_OPT_SMALL_FRONT_NJ, "CHB_SMALL_FRONT_NJ", TILE);
  return v < 0 ? 0 : (v > TILE ? TILE : (int)v);
}

// Small-subtree bundles on (CHB_OPT_SUBTREES = 1, the default) or off (0;
// also CHB_NO_SUBTREES in the environment).
inline bool subtrees_on(const chb_plan& P) {
  if (P.opt[CHB_OPT_SUBTREES] >= 0) return P.opt[CHB_OPT_SUBTREES] != 0;
  return std::getenv("CHB_NO_SUBTREES") == nullptr;
}

// TF32 tiles on tcgen05 (CHB_OPT_TF32_TCGEN05 = 1, or CHB_TF32_TCGEN05 in
// the environment) instead of the warp-level mma.sync tiles (the default).
inline bool tf32_tcgen05(const chb_plan& P) {
  if (P.opt[CHB_OPT_TF32_TCGEN05] >= 0) return P.opt[CHB_OPT_TF32_TCGEN05] != 0;
  return std::getenv("CHB_TF32_TCGEN05") != nullptr;
}

// The triangular solve's additions into vector blocks in a fixed order
// (CHB_OPT_ORDERED_SUMS = 1, or CHB_ORDERED_SUMS in the environment: chains
// of read-modify-write tasks and split-K sums, bit-reproducible) or as
// independent tasks with atomic adds (0, the default: the order of the
// additions, and so the last bits, vary from run to run).
inline bool ordered_sums(const chb_plan& P) {
  if (P.opt[CHB_OPT_ORDERED_SUMS] >= 0) return P.opt[CHB_OPT_ORDERED_SUMS] != 0;
  return std::getenv("CHB_ORDERED_SUMS") != nullptr;
}

// Bytes for the update matrices of cholesky and projected_inverse
// (CHB_OPT_SCRATCH_LIMIT, or CHB_SCRATCH_LIMIT in the environment; -1, the
// default: no limit, each front's update matrix in memory of its own).
inline int64_t scratch_limit_bytes(const chb_plan& P) {
  const int64_t v = plan_option(P, CHB_OPT_SCRATCH_LIMIT, "CHB_SCRATCH_LIMIT", -1);
  return v < 0 ? -1 : v;
}

// Sets a builder up to pool the update matrices under the plan's scratch
// limit (nothing without one, or for a streamed program).  Returns the
// buffer of each front's update matrix (-1: none).
inline std::vector<int> pool_update_matrices(const chb_plan& P, const Program& prog, DagBuilder& B) {
  std::vector<int> buf(P.nsn, -1);
  const int64_t lim = scratch_limit_bytes(P);
  if (lim < 0 || prog.io.in || prog.io.out) return buf;
  B.pool_limit = lim / (int64_t)sizeof(double);
  B.pool_region = P.upd_total;
  // (CHB_SCRATCH_POOL_MIN: smallest pooled update matrix in doubles, default
  // 4096; smaller ones keep their own memory, which keeps the placement's
  // work near (pooled buffers)^2 for trees of many small fronts)
  if (const char* e = std::getenv("CHB_SCRATCH_POOL_MIN")) B.pool_min = std::max<int64_t>(1, std::atoll(e));
  for (int64_t k = 0; k < P.nsn; k++) {
    const FrontDesc& f = P.fronts[k];
    if (f.na > 0) buf[k] = B.pool_buffer(f.upd, (int64_t)f.na * f.na);
  }
  return buf;
}

// After finish(): the program's own supernode descriptors, with the pooled
// offsets of the update matrices.
inline void pooled_fronts(const chb_plan& P, const DagBuilder& B, Program& prog) {
  if (B.pool_limit < 0 || B.pool.empty() || !B.pool_remap) return;
  prog.fronts = P.fronts;
  for (FrontDesc& f : prog.fronts) f.upd = f.na > 0 ? B.pool_remap(f.upd) : 0;
  prog.pool_doubles = B.pool_doubles;
  prog.pool_waits = B.pool_waits;
}

// cholesky's fused diagonal task (CHB_OPT_FUSED_LA = 1, the default where it
// is safe) or separate look-ahead tasks (0; also CHB_NO_FUSED_LA).
inline bool fused_la_allowed(const chb_plan& P) {
  if (P.opt[CHB_OPT_FUSED_LA] >= 0) return P.opt[CHB_OPT_FUSED_LA] != 0;
  return std::getenv("CHB_NO_FUSED_LA") == nullptr;
}

// An operand advanced by k0 along its K dimension.
inline Operand shift_k(Operand o, int k0) {
  switch (o.mode) {
    case OM_N: o.off += (int64_t)k0 * o.ld; break;
    case OM_T: o.off += k0; break;
    case OM_TRI_N: o.off += (int64_t)k0 * o.ld; o.diag -= k0; break;
    case OM_TRI_T: o.off += k0; o.diag += k0; break;
    default: o.pad2 += k0; break;  // OM_SYM: column offset of k = 0
  }
  return o;
}

inline Operand opnd(uint8_t base, int64_t off, int ld, uint8_t mode = OM_N, int diag = 0) {
  Operand o;
  std::memset(&o, 0, sizeof(o));
  o.off = off;
  o.ld = ld;
  o.base = base;
  o.mode = mode;
  o.diag = diag;
  return o;
}

inline Task make_task(uint8_t op) {
  Task t;
  std::memset(&t, 0, sizeof(t));
  t.op = op;
  t.group = -1;
  t.alpha = 1.0;
  t.beta = 0.0;
  return t;
}

inline Task gemm(int m, int n, int k, double alpha, const Operand& a, const Operand& b, double beta,
                 const Operand& c, bool lower = false, int cdiag = 0) {
  Task t = make_task(T_GEMM);
  t.m = m;
  t.n = n;
  t.k = k;
  t.alpha = alpha;
  t.beta = beta;
  t.a = a;
  t.b = b;
  t.c = c;
  t.cmode = lower ? CM_LOWER : CM_FULL;
  t.cdiag = cdiag;
  return t;
}

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace chb

namespace chb {

// A GEMM task split along K into chunks of at most kc: the partial products
// (parts, independent) go to scratch tiles (64 x 64, ld 64, 4096 doubles
// apart, at WS offset `scratch`), and one T_SUM task (`out`) folds them into
// C with the task's alpha, beta and mask.  Waits on the inputs belong on
// every part, waits on C's previous writer on `out` only.  With K <= kc the
// task is emitted as is (parts = {out}).
struct SplitTask {
  std::vector<int> parts;
  int out;
};

inline int split_count(int K, int kc) { return K > kc ? (K + kc - 1) / kc : 1; }

inline SplitTask add_split_gemm(DagBuilder& B, const Task& t, int kc, int64_t scratch, const SchedKey& key,
                                int group = -1) {
  SplitTask st;
  const int p = split_count(t.k, kc);
  if (p == 1) {
    st.out = B.add(t, key, group);
    st.parts.push_back(st.out);
    return st;
  }
  const int chunk = (t.k + p - 1) / p;
  for (int q = 0; q < p; q++) {
    const int k0 = q * chunk, kq = std::min(chunk, t.k - k0);
    Task u = t;
    u.k = kq;
    u.a = shift_k(t.a, k0);
    u.b = shift_k(t.b, k0);
    u.alpha = 1.0;
    u.beta = 0.0;
    u.cmode = CM_FULL;
    u.cdiag = 0;
    u.c = opnd(B_WS, scratch + (int64_t)q * TILE * TILE, TILE);
    SchedKey kk = key;
    kk.rank = key.rank * 64 + q;
    st.parts.push_back(B.add(u, kk));
  }
  Task s = make_task(T_SUM);
  s.m = t.m;
  s.n = t.n;
  s.alpha = t.alpha;
  s.beta = t.beta;
  s.cmode = t.cmode;
  s.cdiag = t.cdiag;
  s.a = opnd(B_WS, scratch, TILE);
  s.c = t.c;
  s.aux[0] = p;
  s.aux[1] = TILE * TILE;
  st.out = B.add(s, key, group, 2.0 + 0.4 * p);
  for (int id : st.parts) B.wait_task(st.out, id);
  return st;
}

// Column groups of the vector extend-add and extract tasks (T_VEC with
// VEC_ASM / VEC_EXTRACT, columns [aux[2], aux[3])): the right-hand sides of
// a front are split so that a task moves about 2,048 elements (sixteen per
// thread, loaded eight at a time), and so that the columns of [x_k; u_k]
// an extend-add stages fit the base shared memory.  Returns the columns per
// task.
inline int vec_cols_per_task(int64_t elems_per_col, int64_t nrhs, int64_t staged_per_col) {
  int64_t g = (elems_per_col * nrhs + 2047) / 2048;
  g = std::max<int64_t>(1, std::min<int64_t>(g, nrhs));
  if (staged_per_col > 0) {
    const int64_t fit = std::max<int64_t>(1, ENGINE_SMEM_BASE_DOUBLES / staged_per_col);
    g = std::max<int64_t>(g, (nrhs + fit - 1) / fit);
  }
  return (int)((nrhs + g - 1) / g);
}

// Small-subtree bundles (T_SUBTREE / T_PSUBTREE).  A subtree qualifies when
// every front in it has nj <= SUB_NJ (and the small-front tasks are on);
// the maximal ones are cut into warp ranges (adjacent subtrees in postorder
// merged up to a modelled cost), four ranges per task.  CHB_OPT_SUBTREES = 0
// (or CHB_NO_SUBTREES) turns bundling off (every small front is then its own T_FRONT / T_PFRONT).
struct Bundles {
  // per task: up to four inclusive ranges [lo, hi] (lo < 0: no range)
  std::vector<std::array<int, 8>> tasks;
  std::vector<int> of;      // supernode -> bundle index, or -1
  std::vector<double> cost; // modelled duration of each bundle (us): its longest range
  std::vector<std::vector<int>> roots;  // per bundle: the supernodes whose parent lies outside it
};

inline double bundle_front_us(const FrontDesc& f) {
  // measured order of magnitude of one warp's front: a fixed part for the
  // loads, pivots and stores, plus the O(nj^2 nn) arithmetic
  return 0.4 + 0.002 * (double)f.nj * f.nj + 0.0004 * (double)f.nj * f.nj * f.nn;
}

inline Bundles make_bundles(const chb_plan& P) {
  Bundles out;
  const int64_t N = P.nsn;
  out.of.assign(N, -1);
  if (!subtrees_on(P) || small_front_nj(P) < SUB_NJ || N == 0) return out;
  std::vector<char> all(N, 1);
  std::vector<int> size(N, 1);
  for (int64_t k = 0; k < N; k++) {
    const FrontDesc& f = P.fronts[k];
    if (f.nj > SUB_NJ) all[k] = 0;
    const int p = f.parent;
    if (p != k && p >= 0 && p < N) {
      all[p] = all[p] && all[k];
      size[p] += size[k];
    }
  }
  // warp ranges: maximal qualifying subtrees in postorder, adjacent ones merged
  const double cap_us = 24.0;
  std::vector<std::array<int, 2>> ranges;
  std::vector<double> rcost;
  for (int64_t k = 0; k < N; k++) {
    const int p = P.fronts[k].parent;
    const bool root = all[k] && (p == k || p < 0 || p >= N || !all[p]);
    if (!root) continue;
    const int lo = (int)(k - size[k] + 1);
    double c = 0.0;
    for (int64_t q = lo; q <= k; q++) c += bundle_front_us(P.fronts[q]);
    if (!ranges.empty() && ranges.back()[1] + 1 == lo && rcost.back() + c <= cap_us) {
      ranges.back()[1] = (int)k;
      rcost.back() += c;
    } else {
      ranges.push_back({lo, (int)k});
      rcost.push_back(c);
    }
  }
  for (size_t r0 = 0; r0 < ranges.size(); r0 += 4) {
    std::array<int, 8> t;
    t.fill(-1);
    double c = 0.0;
    const int b = (int)out.tasks.size();
    out.roots.emplace_back();
    for (size_t w = 0; w < 4 && r0 + w < ranges.size(); w++) {
      t[2 * w] = ranges[r0 + w][0];
      t[2 * w + 1] = ranges[r0 + w][1];
      c = std::max(c, rcost[r0 + w]);
      for (int q = ranges[r0 + w][0]; q <= ranges[r0 + w][1]; q++) {
        out.of[q] = b;
        const int p = P.fronts[q].parent;
        if (p == q || p < 0 || p >= N || p > ranges[r0 + w][1]) out.roots[b].push_back(q);
      }
    }
    out.tasks.push_back(t);
    out.cost.push_back(c);
  }
  return out;
}

// The task of bundle b: op T_SUBTREE or T_PSUBTREE; operands a / b carry the
// [first, end) offsets of the values the bundle touches (for the streamed
// programs' chunk bookkeeping; the device code does not read them).
inline Task bundle_task(const chb_plan& P, const Bundles& bd, int b, uint8_t op) {
  Task t = make_task(op);
  const std::array<int, 8>& r = bd.tasks[b];
  for (int w = 0; w < 4; w++) t.aux[w] = r[2 * w];
  t.m = r[1];
  t.n = r[3];
  t.k = r[5];
  t.cdiag = r[7];
  int64_t lo = INT64_MAX, hi = 0;
  for (int w = 0; w < 4; w++)
    if (r[2 * w] >= 0) {
      lo = std::min<int64_t>(lo, P.fronts[r[2 * w]].blk);
      const FrontDesc& l = P.fronts[r[2 * w + 1]];
      hi = std::max<int64_t>(hi, l.blk + (int64_t)l.nj * l.nn);
    }
  t.a = opnd(B_X, lo, 1);
  t.b = opnd(B_X, hi, 1);
  return t;
}

}  // namespace chb
