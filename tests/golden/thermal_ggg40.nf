%type_of_analysis
0

%type_of_solver
0

%type_of_rhs
0

%voxel_size
1.0

%solver_tolerance
1e-06

%number_of_iterations
1000

%image_dimensions
100 100 100

%refinement
1

%number_of_materials
2

%properties_of_materials
87 129.0
182 80.4

%volume_fraction
11.39 88.61

%data_type
uint8

