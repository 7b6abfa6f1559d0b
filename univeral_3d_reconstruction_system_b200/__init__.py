"""B200-native (sm_100a) 3D Gaussian Splatting trainer: drop-in for the CPU splat core of
Abner0907/univeral_3d_reconstruction_system (engine/src/splat)."""
from .types import (GaussianModel, LearningRates, LossValue, RasterSettings, RenderCamera, TrainImage,  # noqa: F401
                    TrainOptions, TrainStats)
