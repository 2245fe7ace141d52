// ContributionScheduler (reference src/scheduling/contribution_scheduler.cpp
// :23-121): schedule() over hyt_contribution_schedule; the plan bookkeeping
// members follow the reference's definitions on the host.
#include "scheduling/contribution_scheduler.hpp"

#include "hyt/capi.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace hytgraph::scheduling {

std::vector<ContributionPriority> make_contribution_priorities(const std::vector<std::size_t> &item_indices,
                                                               const std::vector<double> &contributions) {
    if (item_indices.size() != contributions.size())
        throw std::invalid_argument("contribution priority inputs must have equal size");
    std::vector<ContributionPriority> p;
    p.reserve(item_indices.size());
    for (std::size_t i = 0; i < item_indices.size(); ++i) p.push_back({item_indices[i], contributions[i]});
    return p;
}

ContributionScheduler::ContributionScheduler(ContributionSchedulerOptions options) : options_(options) {}

ContributionSchedulingPlan ContributionScheduler::schedule(const std::vector<ContributionPriority> &priorities) const {
    ContributionSchedulingPlan plan;
    const std::size_t n = priorities.size();
    plan.metrics.input_item_count = n;
    plan.metrics.scheduled_item_count = n;
    if (n == 0) return plan;
    int devices = 0;
    if (hyt_device_count(&devices) != HYT_OK || devices == 0)
        throw std::runtime_error("ContributionScheduler::schedule: no CUDA device is available");
    std::vector<uint64_t> items(n), ordered(n);
    std::vector<double> c(n);
    for (std::size_t i = 0; i < n; ++i) {
        items[i] = priorities[i].item_index;
        c[i] = priorities[i].contribution;
    }
    hyt_contribution_metrics m{};
    const int status = hyt_contribution_schedule(items.data(), c.data(), n, options_.deterministic_tie_break ? 1 : 0,
                                                 options_.zero_contribution_epsilon, ordered.data(), &m);
    if (status == HYT_E_INVALID) throw std::invalid_argument(hyt_last_error());
    if (status != HYT_OK) throw std::runtime_error(std::string("ContributionScheduler::schedule: ") + hyt_last_error());
    plan.ordered_item_indices.assign(ordered.begin(), ordered.end());
    plan.metrics.reordered_item_count = m.reordered_item_count;
    plan.metrics.zero_contribution_count = m.zero_contribution_count;
    plan.metrics.scheduling_overhead = m.scheduling_overhead;
    plan.metrics.redundant_work_count = m.redundant_work_count;
    return plan;
}

ContributionSchedulingPlan ContributionScheduler::synchronous_reference(
    const std::vector<ContributionPriority> &priorities) {
    ContributionSchedulingPlan plan;
    plan.metrics.input_item_count = priorities.size();
    plan.metrics.scheduled_item_count = priorities.size();
    for (const auto &p : priorities) {
        plan.ordered_item_indices.push_back(p.item_index);
        if (std::abs(p.contribution) == 0.0) ++plan.metrics.zero_contribution_count;
    }
    return plan;
}

ContributionSchedulingMetrics ContributionScheduler::measure_work_metrics(
    const std::vector<ContributionPriority> &priorities) {
    ContributionSchedulingMetrics m;
    m.input_item_count = priorities.size();
    m.scheduled_item_count = priorities.size();
    std::vector<std::size_t> items;
    items.reserve(priorities.size());
    for (const auto &p : priorities) {
        items.push_back(p.item_index);
        if (std::abs(p.contribution) == 0.0) ++m.zero_contribution_count;
    }
    std::sort(items.begin(), items.end());
    for (std::size_t i = 1; i < items.size(); ++i) m.redundant_work_count += items[i] == items[i - 1];
    return m;
}

ContributionSchedulingMetrics ContributionScheduler::measure_work_metrics(
    const std::vector<ContributionPriority> &priorities, const std::vector<ContributionWorkObservation> &observations) {
    ContributionSchedulingMetrics m = measure_work_metrics(priorities);
    for (const auto &o : observations) m.stale_work_count += o.stale ? 1U : 0U;
    return m;
}

std::vector<ContributionPriority> ContributionScheduler::make_contribution_priorities(
    const std::vector<std::size_t> &item_indices, const std::vector<double> &contributions) {
    return scheduling::make_contribution_priorities(item_indices, contributions);
}

double ContributionScheduler::estimate_scheduling_overhead(const std::vector<ContributionPriority> &priorities) {
    return priorities.empty() ? 0.0 : std::log2(static_cast<double>(priorities.size()));
}

}  // namespace hytgraph::scheduling
