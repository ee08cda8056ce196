// kr_template.h -- native body templates of the batched engine.
//
// A template is the constraint graph of one body shape (A arms x S segments)
// with its solve schedule, built exactly as the reference builds a creature:
// spawnKraken's creation order (src/body/kraken.js:64-148), createSim's
// greedy colouring in creation order (src/sim/core.js:45-58 with
// assignColor, src/physics/xpbd.js:98-105), the stable grouping by colour
// (core.js:276-288), and from that list order the body-disjoint levels the
// warp sweeps.  Spawn poses follow the same chain rule (kraken.js:64-101).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace kr {

constexpr int kMaxArms = 8;
constexpr int kMaxSegs = 9;
constexpr int kMaxTplBodies = 1 + kMaxArms * kMaxSegs;            // 73
constexpr int kMaxTplCons = kMaxArms * (2 * kMaxSegs + 1);        // 152
constexpr int kMaxTplPts = 8 + 2 * kMaxArms * kMaxSegs;           // 152
constexpr int kMaxTplLevels = 64;

// Solve schedules per lane-group size: 32, 16 and 8 lanes per creature.
constexpr int kSchedules = 3;
constexpr int schedule_index(int lanes) { return lanes == 32 ? 0 : lanes == 16 ? 1 : 2; }

// One solve schedule of the constraint list: the constraint slots level by
// level (each level body-disjoint and of one constraint type) with their
// static data.
struct Schedule {
  int nlv = 0;
  std::vector<int> lvl;                 // nlv + 1 level offsets
  std::vector<int> ab;                  // local a | local b << 16 (b = 0xffff: world)
  std::vector<int> type;                // 0 pin, 1 angle, 2 grip
  std::vector<int> motor;               // a * segs + j for motor j of arm a, else -1
  std::vector<float> lax, lay, lbx, lby, rest, minA, maxA;
  std::vector<int> arm_grip;            // slot of each arm's grip
};

struct Template {
  int arms = 0, segs = 0;
  int nb = 0, nc = 0, np = 0, nlv = 0;
  // bodies
  std::vector<float> im, ii;            // f32 as uploaded (gpuworld.js:258-259)
  std::vector<int> boff, bcnt;          // collision points per body
  // constraints in schedule order (level by level), as in sched[0]
  std::vector<int> ab;                  // local a | local b << 16 (b = 0xffff: world)
  std::vector<int> type;                // 0 pin, 1 angle, 2 grip
  std::vector<float> lax, lay, lbx, lby, rest, minA, maxA;
  std::vector<int> motor;               // a * segs + j for motor j of arm a, else -1
  std::vector<int> lvl;                 // nlv + 1 level offsets
  // per lane-group size (schedule_index): the same constraints in levels
  // balanced for that many lanes
  Schedule sched[kSchedules];
  // collision points grouped per body in creation order
  std::vector<float> plx, ply, pr;
  std::vector<int> pbody;
  // arms
  std::vector<int> arm_tip;             // tip body
  std::vector<int> arm_grip;            // schedule slot of the grip
  std::vector<int> arm_seg0;            // first segment body
  std::vector<int> arm_segs;            // arms x segs body ids
  float r_max = 0.f;                    // largest collision radius
  float off_max = 0.f;                  // largest distance of a collision point from its body's centre
  double reach = 0.0;                   // ARM_REACH for this segment count
};

// Builds the template of an arms x segs body; returns false with a message
// if the shape is out of range.
bool build_template(int arms, int segs, Template *t, std::string *err);

// spawnKraken's pose (kraken.js:64-101): body positions and angles of a
// creature spawned at (x, y, angle), in f64, body order of the template.
void spawn_pose(const Template &t, double x, double y, double angle, double curl, double *px,
                double *py, double *ang);

}  // namespace kr
