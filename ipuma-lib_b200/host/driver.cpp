#include "driver.hpp"

#include <mutex>
#include <stdexcept>

static ipu::batchaffine::SWAlgorithm* g_driver = nullptr;
static std::mutex g_driver_mutex;

ipu::batchaffine::SWAlgorithm* getDriver() {
  std::lock_guard<std::mutex> lk(g_driver_mutex);
  if (!g_driver) throw std::runtime_error("init_single_ipu has not been called");
  return g_driver;
}

void init_single_ipu(ipu::SWConfig config, ipu::IPUAlgoConfig algoconfig) {
  std::lock_guard<std::mutex> lk(g_driver_mutex);
  if (!g_driver) g_driver = new ipu::batchaffine::SWAlgorithm(config, algoconfig, 0);
}
