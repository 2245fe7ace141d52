#pragma once
// Contribution-driven work ordering.  Source-compatible with
// hytgraph::scheduling::ContributionScheduler (reference
// include/scheduling/contribution_scheduler.hpp,
// src/scheduling/contribution_scheduler.cpp:23-121): items by descending
// contribution, ties by lower item index (or input order), with the plan
// metrics.  schedule() runs on the GPU (hyt_contribution_schedule) and
// throws std::runtime_error when no CUDA device is available; the other
// members are plan bookkeeping on the host.

#include <cstddef>
#include <vector>

namespace hytgraph::scheduling {

enum class ContributionSchedulingPolicy { PageRankDelta, SSSPContribution };

struct ContributionPriority {
    std::size_t item_index = 0U;
    double contribution = 0.0;
};

struct ContributionSchedulingMetrics {
    std::size_t input_item_count = 0U;
    std::size_t scheduled_item_count = 0U;
    std::size_t reordered_item_count = 0U;
    std::size_t zero_contribution_count = 0U;
    double scheduling_overhead = 0.0;
    std::size_t stale_work_count = 0U;
    std::size_t redundant_work_count = 0U;
};

struct ContributionSchedulingPlan {
    std::vector<std::size_t> ordered_item_indices;
    ContributionSchedulingMetrics metrics;
    [[nodiscard]] std::size_t size() const noexcept { return ordered_item_indices.size(); }
    [[nodiscard]] bool empty() const noexcept { return ordered_item_indices.empty(); }
    [[nodiscard]] bool reordered() const noexcept { return metrics.reordered_item_count != 0U; }
};

struct ContributionSchedulerOptions {
    ContributionSchedulingPolicy policy = ContributionSchedulingPolicy::PageRankDelta;
    bool deterministic_tie_break = true;
    double zero_contribution_epsilon = 0.0;
};

struct ContributionWorkObservation {
    std::size_t item_index = 0U;
    bool stale = false;
};

[[nodiscard]] std::vector<ContributionPriority> make_contribution_priorities(
    const std::vector<std::size_t> &item_indices, const std::vector<double> &contributions);

class ContributionScheduler {
public:
    explicit ContributionScheduler(ContributionSchedulerOptions options = {});
    [[nodiscard]] const ContributionSchedulerOptions &options() const noexcept { return options_; }
    // Throws std::invalid_argument for a non-finite contribution.
    [[nodiscard]] ContributionSchedulingPlan schedule(const std::vector<ContributionPriority> &priorities) const;
    [[nodiscard]] static ContributionSchedulingPlan synchronous_reference(
        const std::vector<ContributionPriority> &priorities);
    [[nodiscard]] static ContributionSchedulingMetrics measure_work_metrics(
        const std::vector<ContributionPriority> &priorities);
    [[nodiscard]] static ContributionSchedulingMetrics measure_work_metrics(
        const std::vector<ContributionPriority> &priorities,
        const std::vector<ContributionWorkObservation> &observations);
    [[nodiscard]] std::vector<ContributionPriority> make_contribution_priorities(
        const std::vector<std::size_t> &item_indices, const std::vector<double> &contributions);
    [[nodiscard]] static double estimate_scheduling_overhead(const std::vector<ContributionPriority> &priorities);

private:
    ContributionSchedulerOptions options_;
};

}  // namespace hytgraph::scheduling
