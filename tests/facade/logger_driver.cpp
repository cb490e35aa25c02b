// logger of include/exafmm_b200.hpp without a solve, for tests/test_facade.py:
// two events timed around short sleeps (one twice), written with writeTime to
// the directory given as the argument (optional second argument: the name
// field's width, logger::stringLength), then a second writeTime after reset.
#include <chrono>
#include <thread>

#include "exafmm_b200.hpp"
using namespace exafmm_laplace;

int main(int argc, char **argv) {
  if (argc < 2) return 2;
  logger::path = argv[1];
  if (argc > 2) logger::stringLength = std::atoi(argv[2]);
  for (int i = 0; i < 2; i++) {
    logger::startTimer("Total FMM");
    std::this_thread::sleep_for(std::chrono::milliseconds(30));
    logger::stopTimer("Total FMM");
  }
  logger::startTimer("Direct sum");
  std::this_thread::sleep_for(std::chrono::milliseconds(20));
  logger::stopTimer("Direct sum");
  logger::writeTime(2);
  logger::startTimer("Total FMM");
  logger::stopTimer("Total FMM");
  logger::resetTimer();
  logger::writeTime(3);
  return 0;
}
