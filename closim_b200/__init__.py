"""closim_b200: the implicit-Euler Newton cloth step of mohdabraralikhan/closim
as a B200-native CUDA solver behind the reference's ClothSolver interface."""
from .solver import (ClothMaterial, ClothMeshData, ClothScene, ClothSolverError, ContactParams, ContactSystem,
                     CudaSolver, DEFAULT_CONTACT_PARAMS, DEFAULT_MATERIAL, StepStats, buildGrid, createScene,
                     enforcePins, pinColumn, preprocess)

__all__ = ["ClothMaterial", "ClothMeshData", "ClothScene", "ClothSolverError", "ContactParams", "ContactSystem",
           "CudaSolver", "DEFAULT_CONTACT_PARAMS", "DEFAULT_MATERIAL", "StepStats", "buildGrid", "createScene",
           "enforcePins", "pinColumn", "preprocess"]
