%type_of_analysis
2

%type_of_solver
0

%type_of_rhs
0

%voxel_size
0.01

%solver_tolerance
1e-06

%number_of_iterations
5000

%image_dimensions
100 100 0

%refinement
1

%number_of_materials
2

%properties_of_materials
0
255

%volume_fraction
88.89 11.11

%data_type
uint8

