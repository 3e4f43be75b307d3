// Library-wide count of kernel launches (read by fdtd_launch_count).
#pragma once

namespace fdtd {
void count_launches(int n);
}  // namespace fdtd
