// multi.cpp -- one batch spread over several devices.
//
// Frames are independent (src/pool.rs:3-8; the crate leaves frame-level
// parallelism to its caller, src/decode.rs:15-17), so a batch splits by
// frame with no exchange between devices: each device codes its share in
// one batched call of its own context, on a host thread of its own, and the
// results are put back in input order. Shares are balanced by macroblock
// count, the work a frame costs.

#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "../../include/prores_b200.h"
#include "engine.h"

namespace prores {
namespace {

uint64_t macroblocks(uint32_t w, uint32_t h) { return (uint64_t)((w + 15u) / 16u) * ((h + 15u) / 16u); }

// Largest frames first, each to the part with the fewest macroblocks so far
// (ties to the lower part); a frame of weight 0 goes to part 0.
void shard(const std::vector<uint64_t> &weight, int parts, std::vector<int> &part) {
    const int n = (int)weight.size();
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return weight[a] > weight[b]; });
    std::vector<uint64_t> load(parts, 0);
    part.assign(n, 0);
    for (int i : order) {
        int best = 0;
        for (int k = 1; k < parts; k++)
            if (load[k] < load[best]) best = k;
        part[i] = best;
        load[best] += weight[i];
    }
}

// What a part's call left behind: its return code, its thread's last error
// and per-frame messages (those are thread-local).
struct PartResult {
    int code = PRORES_OK;
    std::string last;
    std::vector<std::string> msgs;
};

template <class Call>
int run_parts(int parts, const std::vector<std::vector<int>> &members, std::vector<PartResult> &res, Call call) {
    res.assign(parts, PartResult{});
    std::vector<std::thread> threads;
    auto work = [&](int p) {
        if (members[p].empty()) return;
        res[p].code = call(p);
        res[p].last = prores_last_error();
        res[p].msgs.resize(members[p].size());
        for (size_t k = 0; k < members[p].size(); k++) res[p].msgs[k] = prores_batch_error((int)k);
    };
    for (int p = 1; p < parts; p++) threads.emplace_back(work, p);
    work(0);
    for (auto &t : threads) t.join();
    for (int p = 0; p < parts; p++)
        if (!members[p].empty() && res[p].code != PRORES_OK) return p;
    return -1;
}

int finish_parts(const std::vector<std::vector<int>> &members, const std::vector<PartResult> &res, int failed,
                 int n, const int *status) {
    if (failed >= 0) {
        set_last_error_text(res[failed].last);
        return res[failed].code;
    }
    // Each frame's message, in input order, and the first failing frame's as
    // the last error, as a one-device batch leaves them.
    std::vector<std::string> msgs(n);
    int first = -1;
    for (size_t p = 0; p < members.size(); p++)
        for (size_t k = 0; k < members[p].size(); k++) {
            const int i = members[p][k];
            if (status[i] != PRORES_OK) {
                msgs[i] = res[p].msgs[k];
                if (first < 0 || i < first) first = i;
            }
        }
    set_batch_error_texts(msgs);
    if (first >= 0) set_last_error_text(msgs[first]);
    return PRORES_OK;
}

}  // namespace
}  // namespace prores

using namespace prores;

extern "C" {

int prores_shard_frames(const uint32_t *width, const uint32_t *height, int n, int parts, int *part) {
    if (n < 0 || parts < 1 || (n && (!width || !height || !part))) {
        set_last_error(make_status(PRORES_CONFIG, "no frames or parts"));
        return PRORES_CONFIG;
    }
    std::vector<uint64_t> w(n);
    for (int i = 0; i < n; i++) w[i] = macroblocks(width[i], height[i]);
    std::vector<int> p;
    shard(w, parts, p);
    std::copy(p.begin(), p.end(), part);
    return PRORES_OK;
}

int prores_decode_batch_multi(prores_ctx *const *ctxs, int n_ctx, const prores_buf *in, int n,
                              uint32_t out_bit_depth, prores_frame *out, int *status) {
    if (!ctxs || n_ctx < 1 || n < 0 || (n && (!in || !out || !status))) {
        set_last_error(make_status(PRORES_CONFIG, "no contexts or frames"));
        return PRORES_CONFIG;
    }
    for (int k = 0; k < n_ctx; k++)
        if (!ctxs[k]) {
            set_last_error(make_status(PRORES_CONFIG, "no context"));
            return PRORES_CONFIG;
        }
    // Weights from the frame headers; a frame whose header fails costs
    // nothing on the device (its error comes from the host).
    std::vector<uint64_t> weight(n, 0);
    for (int i = 0; i < n; i++) {
        prores_frame info;
        if (!probe_frame(in[i].data, in[i].len, out_bit_depth, &info))
            weight[i] = macroblocks(info.width, info.height);
    }
    std::vector<int> part;
    shard(weight, n_ctx, part);
    std::vector<std::vector<int>> members(n_ctx);
    for (int i = 0; i < n; i++) members[part[i]].push_back(i);
    std::vector<std::vector<prores_buf>> ins(n_ctx);
    std::vector<std::vector<prores_frame>> outs(n_ctx);
    std::vector<std::vector<int>> stats(n_ctx);
    for (int p = 0; p < n_ctx; p++) {
        for (int i : members[p]) {
            ins[p].push_back(in[i]);
            outs[p].push_back(out[i]);
        }
        stats[p].assign(members[p].size(), PRORES_OK);
    }
    std::vector<PartResult> res;
    const int failed = run_parts(n_ctx, members, res, [&](int p) {
        return prores_decode_batch(ctxs[p], ins[p].data(), (int)ins[p].size(), out_bit_depth, outs[p].data(),
                                   stats[p].data());
    });
    for (int p = 0; p < n_ctx; p++)
        for (size_t k = 0; k < members[p].size(); k++) {
            out[members[p][k]] = outs[p][k];
            status[members[p][k]] = stats[p][k];
        }
    return finish_parts(members, res, failed, n, status);
}

int prores_encode_batch_multi(prores_ctx *const *ctxs, int n_ctx, const prores_config *cfg, const prores_frame *in,
                              int n, prores_buf *out, int *status) {
    if (!ctxs || n_ctx < 1 || n < 0 || (n && (!cfg || !in || !out || !status))) {
        set_last_error(make_status(PRORES_CONFIG, "no contexts or frames"));
        return PRORES_CONFIG;
    }
    for (int k = 0; k < n_ctx; k++)
        if (!ctxs[k]) {
            set_last_error(make_status(PRORES_CONFIG, "no context"));
            return PRORES_CONFIG;
        }
    std::vector<uint64_t> weight(n);
    for (int i = 0; i < n; i++) weight[i] = macroblocks(in[i].width, in[i].height);
    std::vector<int> part;
    shard(weight, n_ctx, part);
    std::vector<std::vector<int>> members(n_ctx);
    for (int i = 0; i < n; i++) members[part[i]].push_back(i);
    std::vector<std::vector<prores_config>> cfgs(n_ctx);
    std::vector<std::vector<prores_frame>> ins(n_ctx);
    std::vector<std::vector<prores_buf>> outs(n_ctx);
    std::vector<std::vector<int>> stats(n_ctx);
    for (int p = 0; p < n_ctx; p++) {
        for (int i : members[p]) {
            cfgs[p].push_back(cfg[i]);
            ins[p].push_back(in[i]);
        }
        outs[p].assign(members[p].size(), prores_buf{nullptr, 0});
        stats[p].assign(members[p].size(), PRORES_OK);
    }
    std::vector<PartResult> res;
    const int failed = run_parts(n_ctx, members, res, [&](int p) {
        return prores_encode_batch(ctxs[p], cfgs[p].data(), ins[p].data(), (int)ins[p].size(), outs[p].data(),
                                   stats[p].data());
    });
    if (failed >= 0) {
        // A device failure on one part fails the call: no packet is handed out.
        for (int p = 0; p < n_ctx; p++)
            for (auto &b : outs[p]) free(const_cast<uint8_t *>(b.data));
        for (int i = 0; i < n; i++) out[i] = prores_buf{nullptr, 0};
    } else {
        for (int p = 0; p < n_ctx; p++)
            for (size_t k = 0; k < members[p].size(); k++) {
                out[members[p][k]] = outs[p][k];
                status[members[p][k]] = stats[p][k];
            }
    }
    return finish_parts(members, res, failed, n, status);
}

}  // extern "C"
