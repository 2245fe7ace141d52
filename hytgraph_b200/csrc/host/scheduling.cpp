// TaskCombiner: per-partition engine decisions -> executable tasks, with the
// grouping rules of the reference (src/scheduling/task_combiner.cpp:67-248).
#include "scheduling/task_combiner.hpp"

#include <algorithm>
#include <stdexcept>

namespace hytgraph::scheduling {

using transfer::TransferEngine;

TaskCombiner::TaskCombiner(TaskCombinerOptions options) : options_(options) {
    if (options_.filter_combine_k == 0U)
        throw std::invalid_argument("TaskCombiner: filter_combine_k must be greater than zero");
}

namespace {
ExecutableTask task_of(TransferEngine engine, std::vector<std::size_t> members) {
    ExecutableTask t;
    t.engine = engine;
    if (!members.empty()) {
        t.first_partition_index = members.front();
        t.end_partition_index = members.back() + 1U;
    }
    t.partition_indices = std::move(members);
    return t;
}
}  // namespace

TaskCombinationPlan TaskCombiner::combine(const std::vector<TransferEngine> &engines) const {
    if (options_.filter_combine_k == 0U)
        throw std::invalid_argument("TaskCombiner: filter_combine_k must be greater than zero");
    TaskCombinationPlan plan;
    plan.metrics.logical_partition_count = engines.size();
    std::vector<ExecutableTask> tasks;
    std::vector<std::size_t> compaction, zero_copy;
    for (std::size_t i = 0; i < engines.size();) {
        switch (engines[i]) {
            case TransferEngine::ExpTMFilter: {
                std::vector<std::size_t> group;
                while (i < engines.size() && engines[i] == TransferEngine::ExpTMFilter &&
                       group.size() < options_.filter_combine_k)
                    group.push_back(i++);
                tasks.push_back(task_of(TransferEngine::ExpTMFilter, std::move(group)));
                break;
            }
            case TransferEngine::ExpTMCompaction: compaction.push_back(i++); break;
            case TransferEngine::ImpTMZeroCopy: zero_copy.push_back(i++); break;
            default: throw std::invalid_argument("TaskCombiner: unsupported transfer engine");
        }
    }
    if (!compaction.empty()) tasks.push_back(task_of(TransferEngine::ExpTMCompaction, std::move(compaction)));
    if (!zero_copy.empty()) tasks.push_back(task_of(TransferEngine::ImpTMZeroCopy, std::move(zero_copy)));
    std::stable_sort(tasks.begin(), tasks.end(), [](const ExecutableTask &a, const ExecutableTask &b) {
        return a.first_partition_index < b.first_partition_index;
    });
    for (std::size_t k = 0; k < tasks.size(); ++k) {
        ExecutableTask &t = tasks[k];
        t.task_index = k;
        const std::size_t n = t.partition_count();
        if (t.engine == TransferEngine::ExpTMFilter) {
            if (n > 1U) plan.metrics.filter_partitions_combined += n - 1U;
        } else if (t.engine == TransferEngine::ExpTMCompaction) {
            plan.metrics.compaction_partitions_combined += n;
        } else {
            plan.metrics.zero_copy_partitions_combined += n;
        }
    }
    plan.metrics.executable_task_count = tasks.size();
    plan.tasks = std::move(tasks);
    return plan;
}

}  // namespace hytgraph::scheduling
