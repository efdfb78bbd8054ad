"""Three eager MIXED stage-1 steps (128 antennas x 2048 rays x 128 target samples,
64 coarse, S = 256) for an ncu launch list:

    ncu --metrics gpu__time_duration.sum --clock-control none -c 8000 --csv \\
        --log-file launches_stage1.csv python -m benchkit.stage1_profile
"""
from __future__ import annotations


def main() -> int:
    import torch

    from .stage1 import Stage1RFStep

    st = Stage1RFStep(num_antennas=128, num_rays=2048, samples_per_ray=128, num_adc=256, precision="mixed",
                      seed=0)
    for _ in range(3):
        st.resample()
        st.run()
    torch.cuda.synchronize()
    print("ok")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
