#pragma once
// Groups per-partition engine decisions into executable tasks.
// Source-compatible with hytgraph::scheduling::TaskCombiner (reference
// include/scheduling/task_combiner.hpp:17-163).  The executing engine uses
// the task list as its per-iteration launch/copy schedule: each Filter task
// is one copy + kernel pass, the Compaction task one gather + copy + kernel,
// the Zero-Copy task one mapped-read kernel.

#include "transfer/hytm_cost_model.hpp"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace hytgraph::scheduling {

struct ExecutableTask {
    std::size_t task_index = 0U;
    transfer::TransferEngine engine = transfer::TransferEngine::ExpTMFilter;
    std::vector<std::size_t> partition_indices;  // authoritative membership
    std::size_t first_partition_index = 0U;
    std::size_t end_partition_index = 0U;        // last member + 1
    [[nodiscard]] std::size_t partition_count() const noexcept { return partition_indices.size(); }
    [[nodiscard]] bool empty() const noexcept { return partition_indices.empty(); }
};

struct TaskCombinationMetrics {
    std::size_t logical_partition_count = 0U;
    std::size_t executable_task_count = 0U;
    std::size_t filter_partitions_combined = 0U;
    std::size_t compaction_partitions_combined = 0U;
    std::size_t zero_copy_partitions_combined = 0U;
    [[nodiscard]] bool task_count_reduced() const noexcept { return executable_task_count < logical_partition_count; }
    [[nodiscard]] std::size_t task_count_reduction() const noexcept {
        return logical_partition_count >= executable_task_count ? logical_partition_count - executable_task_count : 0U;
    }
};

struct TaskCombinationPlan {
    std::vector<ExecutableTask> tasks;
    TaskCombinationMetrics metrics;
    [[nodiscard]] std::size_t executable_task_count() const noexcept { return tasks.size(); }
};

struct TaskCombinerOptions {
    std::size_t filter_combine_k = 4U;  // max consecutive Filter partitions per task
};

class TaskCombiner {
public:
    // Throws std::invalid_argument when filter_combine_k == 0.
    explicit TaskCombiner(TaskCombinerOptions options = {});
    [[nodiscard]] const TaskCombinerOptions &options() const noexcept { return options_; }
    // Consecutive Filter partitions -> tasks of <= k; all Compaction
    // partitions -> one task; all Zero-Copy partitions -> one task; tasks
    // ordered by their first partition.
    [[nodiscard]] TaskCombinationPlan combine(const std::vector<transfer::TransferEngine> &partition_engines) const;

private:
    TaskCombinerOptions options_;
};

}  // namespace hytgraph::scheduling
