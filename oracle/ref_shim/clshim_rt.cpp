// Runtime of the OpenCL C -> C++ shim: NDRange execution on host threads, with
// barrier() implemented by switching between per-work-item user contexts.
#include "clshim.hpp"

#include <omp.h>

#include <cstdio>
#include <cstdlib>
#include <functional>

namespace clshim {

thread_local WorkItem* cur_item = nullptr;
thread_local const NDRange* cur_range = nullptr;

namespace {
struct GroupRun {
  ucontext_t sched;
  std::vector<ucontext_t> ctx;
  std::vector<WorkItem> items;
  std::vector<char> done;
  std::vector<char> stacks;
  const std::function<void()>* body;
  int current;
};
thread_local GroupRun* cur_group = nullptr;

void item_entry(int idx) {
  GroupRun* g = cur_group;
  (*g->body)();
  g->done[idx] = 1;
  swapcontext(&g->ctx[idx], &g->sched);
}
}  // namespace

void barrier_impl() {
  GroupRun* g = cur_group;
  if (!g) return;  // non-cooperative launch: items run alone, nothing to wait for
  int i = g->current;
  swapcontext(&g->ctx[i], &g->sched);
}

void run_ndrange_fn(int dims, const size_t* gsz, const size_t* lsz_in, bool cooperative,
                    const std::function<void()>& body) {
  NDRange R;
  R.dims = dims;
  for (int d = 0; d < 3; ++d) {
    R.gsz[d] = d < dims ? gsz[d] : 1;
    R.lsz[d] = (d < dims && lsz_in) ? lsz_in[d] : 1;
    if (R.gsz[d] % R.lsz[d]) {
      fprintf(stderr, "clshim: global size not a multiple of local size\n");
      abort();
    }
  }
  const size_t ng[3] = {R.gsz[0] / R.lsz[0], R.gsz[1] / R.lsz[1], R.gsz[2] / R.lsz[2]};
  const long ngroups = (long)(ng[0] * ng[1] * ng[2]);
  const size_t L = R.lsz[0] * R.lsz[1] * R.lsz[2];
#pragma omp parallel
  {
    cur_range = &R;
    GroupRun g;
    const size_t stack_sz = 64 * 1024;
    if (cooperative) {
      g.ctx.resize(L);
      g.items.resize(L);
      g.done.resize(L);
      g.stacks.resize(L * stack_sz);
      g.body = &body;
    }
#pragma omp for schedule(dynamic, 1)
    for (long gi = 0; gi < ngroups; ++gi) {
      size_t gp[3] = {(size_t)gi % ng[0], ((size_t)gi / ng[0]) % ng[1], (size_t)gi / (ng[0] * ng[1])};
      if (!cooperative) {
        WorkItem it;
        cur_item = &it;
        for (size_t l = 0; l < L; ++l) {
          size_t lp[3] = {l % R.lsz[0], (l / R.lsz[0]) % R.lsz[1], l / (R.lsz[0] * R.lsz[1])};
          for (int d = 0; d < 3; ++d) {
            it.lid[d] = lp[d];
            it.grp[d] = gp[d];
            it.gid[d] = gp[d] * R.lsz[d] + lp[d];
          }
          body();
        }
        continue;
      }
      cur_group = &g;
      for (size_t l = 0; l < L; ++l) {
        size_t lp[3] = {l % R.lsz[0], (l / R.lsz[0]) % R.lsz[1], l / (R.lsz[0] * R.lsz[1])};
        WorkItem& it = g.items[l];
        for (int d = 0; d < 3; ++d) {
          it.lid[d] = lp[d];
          it.grp[d] = gp[d];
          it.gid[d] = gp[d] * R.lsz[d] + lp[d];
        }
        g.done[l] = 0;
        getcontext(&g.ctx[l]);
        g.ctx[l].uc_stack.ss_sp = g.stacks.data() + l * stack_sz;
        g.ctx[l].uc_stack.ss_size = stack_sz;
        g.ctx[l].uc_link = nullptr;
        makecontext(&g.ctx[l], (void (*)())item_entry, 1, (int)l);
      }
      // round-robin: every item runs until its next barrier (or its end), then the next
      for (;;) {
        bool any = false;
        for (size_t l = 0; l < L; ++l) {
          if (g.done[l]) continue;
          any = true;
          g.current = (int)l;
          cur_item = &g.items[l];
          swapcontext(&g.sched, &g.ctx[l]);
        }
        if (!any) break;
      }
      cur_group = nullptr;
    }
  }
}

}  // namespace clshim
