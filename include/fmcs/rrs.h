// fmcs/rrs.h -- Recursive Random Search (Ye and Kalyanaraman, "A recursive
// random search algorithm for large-scale network parameter configuration",
// SIGMETRICS 2003), the black-box optimizer the reference uses to enumerate
// massaging plans (reference: src/rrs.h:22-191, same template interface).
//
// The algorithm: draw n = ceil(ln(1-p)/ln(1-r)) random points and keep the
// best; then alternate EXPLOITATION (sample the neighbourhood of the current
// best point; after l = ceil(ln(1-q)/ln(1-v)) failures shrink the
// neighbourhood by c, until it is below st) and EXPLORATION (draw one random
// point; if it beats the running threshold -- the mean of the best cost seen
// in each block of n explorations -- exploit around it), until the stop
// criterion holds.
#pragma once

#include <cmath>
#include <cstddef>
#include <random>
#include <vector>

namespace multiAttrSort {

template <class PointType, class CostType>
class RRS {
  public:
    RRS(double p, double r, double q, double v, double c, double st)
        : p_(p), r_(r), q_(q), v_(v), c_(c), st_(st), gen_(0x5EED), dice_(0.0, 1.0)
    {
    }
    virtual ~RRS() {}

    void Optimize()
    {
        const size_t n = (size_t)std::ceil(std::log(1.0 - p_) / std::log(1.0 - r_));
        const size_t l = (size_t)std::ceil(std::log(1.0 - q_) / std::log(1.0 - v_));
        // initial sampling
        best_point_ = GetRandomSample();
        best_cost_ = GetCost(best_point_);
        for (size_t i = 1; i < n; ++i) {
            PointType x = GetRandomSample();
            CostType cx = GetCost(x);
            if (cx < best_cost_) {
                best_cost_ = cx;
                best_point_ = x;
            }
        }
        PointType explore_best = best_point_;
        CostType explore_cost = best_cost_;
        std::vector<CostType> block_best{best_cost_};
        CostType threshold = best_cost_;
        bool exploit = true;
        size_t explored = 0;
        while (!StopCritera()) {
            if (exploit) {
                PointType center = explore_best;
                CostType center_cost = GetCost(center);
                double rho = r_;
                size_t fails = 0;
                while (rho > st_ && !StopCritera()) {
                    PointType x = GetRandomNeighbor(center, rho);
                    CostType cx = GetCost(x);
                    if (cx < center_cost) {
                        center = x;
                        center_cost = cx;
                        fails = 0;
                    } else if (++fails == l) {
                        rho *= c_;
                        fails = 0;
                    }
                }
                if (center_cost < best_cost_) {
                    best_cost_ = center_cost;
                    best_point_ = center;
                }
                exploit = false;
            }
            PointType x = GetRandomSample();
            CostType cx = GetCost(x);
            if (cx < explore_cost) {
                explore_best = x;
                explore_cost = cx;
            }
            if (cx < threshold) exploit = true;
            if (++explored == n) {
                block_best.push_back(explore_cost);
                CostType sum = CostType(0);
                for (const CostType &b : block_best) sum += b;
                threshold = sum / (CostType)block_best.size();
                explored = 0;
            }
        }
    }

    PointType GetOptimalPoint() { return best_point_; }
    CostType GetOptimalCost() { return best_cost_; }

  protected:
    virtual PointType GetRandomSample() = 0;
    virtual CostType GetCost(const PointType &point) = 0;
    virtual bool StopCritera() = 0;
    virtual PointType GetRandomNeighbor(const PointType &point, double ro) = 0;
    double Dice() { return dice_(gen_); }

  private:
    double p_, r_, q_, v_, c_, st_;
    std::mt19937_64 gen_;
    std::uniform_real_distribution<double> dice_;
    PointType best_point_;
    CostType best_cost_ = CostType(0);
};

}  // namespace multiAttrSort
